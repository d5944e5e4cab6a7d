"""Host-side scene and file output: the TubeSet form of the generator, OBJ/MTL
and PNG writers (no GPU)."""
import os
import zlib

import numpy as np

from lsystemeditor_b200.export import read_obj_triangles, write_obj, write_png
from lsystemeditor_b200.records import MATERIAL_DTYPE, default_material
from lsystemeditor_b200.scene import (HostMesh, TubeSet, batch_scenes, leaf_quads, loft, quad_mesh, refine_segments,
                                      stochastic_tree, tree_tubes)


def test_tubeset_host_mesh_is_the_generator_mesh():
    segs, leaves = stochastic_tree(iterations=4, seed=3)
    segs = refine_segments(segs, 5, taper=0.8)
    ground = quad_mesh((0, 0, 0), (4, 0, 0), (0, 0, -4), default_material(r=0.5, g=0.5, b=0.5))
    bank = HostMesh.empty()
    bank.materials = np.array([default_material(r=0.3), default_material(r=0.1, g=0.5)], MATERIAL_DTYPE)
    extra = HostMesh.concat([bank, ground])
    ts = TubeSet.from_turtle(segs, leaves, 12, 0.2, leaf_material=1, extra=extra)
    a = ts.host_mesh()
    tube = loft(segs, 12)
    leaf = leaf_quads(leaves, 0.2, 0)
    leaf.materials = bank.materials[1:2]
    tube.materials = bank.materials[0:1]
    b = HostMesh.concat([tube, leaf, ground])
    assert a.triangle_count == ts.triangle_count == b.triangle_count
    for f in ("positions", "normals", "uvs", "material_ids"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert len(a.materials) == 3


def test_batch_workload_draws():
    tubes, cams, sizes, params = batch_scenes(count=6, sides=8, rings=4)
    assert len(tubes) == len(cams) == len(sizes) == 6
    assert all(w == h and w in (256, 512, 768, 1024) for w, h in sizes)
    assert int(params["max_samples_per_pixel"]) == 512 and int(params["adaptive_criterion"]) == 1
    again = batch_scenes(count=6, sides=8, rings=4)
    assert all(np.array_equal(x.points, y.points) for x, y in zip(tubes, again[0]))


def test_write_obj_round_trip(tmp_path):
    ts = tree_tubes(iterations=3, seed=1, sides=6, rings=3)
    mesh = ts.host_mesh()
    path = os.path.join(tmp_path, "tree.obj")
    write_obj(path, mesh)
    tri, mats = read_obj_triangles(path)
    assert tri.shape == (mesh.triangle_count, 3, 3)
    assert np.allclose(tri, mesh.positions, atol=1e-6)
    assert mats[0] == "mat_0" and mats[-1] == f"mat_{int(mesh.material_ids[-1])}"
    mtl = open(os.path.join(tmp_path, "tree.mtl")).read()
    assert mtl.count("newmtl mat_") == len(mesh.materials) == 4
    # the light (material 3) is emissive: Ke = Kd x emission
    assert "Ke 10.000000 10.000000 10.000000" in mtl
    # bark roughness 0.8 -> Ns = 10 + (1 - 0.8) * 990 in single precision
    ns = np.float32(10.0) + (np.float32(1.0) - np.float32(0.8)) * np.float32(990.0)
    assert f"Ns {float(ns):.6f}" in mtl and abs(float(ns) - 208.0) < 1e-3


def test_write_png(tmp_path):
    img = np.zeros((3, 5, 4), np.uint8)
    img[..., 0] = np.arange(5)[None, :] * 50
    img[..., 3] = 255
    path = os.path.join(tmp_path, "a.png")
    write_png(path, img)
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    n = int.from_bytes(data[8:12], "big")
    assert data[12:16] == b"IHDR" and int.from_bytes(data[16:20], "big") == 5 and int.from_bytes(data[20:24], "big") == 3
    idat = data.index(b"IDAT")
    ln = int.from_bytes(data[idat - 4:idat], "big")
    raw = zlib.decompress(data[idat + 4:idat + 4 + ln])
    rows = [raw[r * 21 + 1:(r + 1) * 21] for r in range(3)]
    assert np.array_equal(np.frombuffer(b"".join(rows), np.uint8).reshape(3, 5, 4), img)
    assert n == 13
