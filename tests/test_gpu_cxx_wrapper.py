"""The C++ PathTracer-shaped wrapper (tests/cpp/PathTracerB200.h), compiled
against the reference's own headers (HostMesh, CameraGpu, RenderParamsGpu,
MaterialGpu; its static_asserts pin the record layouts at compile time) and
linked to libpt_b200.so, renders the same image as the Python binding: the
reference's records pass through the C ABI unchanged."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from lsystemeditor_b200.records import default_params
from tests.helpers import zoo_camera, zoo_scene

pytestmark = pytest.mark.gpu


def test_cxx_wrapper_renders_like_the_python_binding(tracer):
    from oracle.bindings import WRAPPER_BIN
    if not os.path.exists(WRAPPER_BIN):
        pytest.skip("the C++ wrapper check was not built (no reference headers where build() ran)")
    mesh = zoo_scene(n_per_mat=60, seed=4).contiguous()
    w, h, spp = 40, 32, 4
    cam = zoo_camera(w, h)
    with tempfile.TemporaryDirectory() as tmp:
        scene, image = os.path.join(tmp, "scene.bin"), os.path.join(tmp, "image.bin")
        with open(scene, "wb") as f:
            textures = mesh.textures if mesh.textures is not None else np.zeros(0, np.uint8)
            np.array([w, h, spp, mesh.triangle_count, len(mesh.materials), len(textures)], np.int32).tofile(f)
            tri = np.concatenate([mesh.positions.reshape(-1, 9), mesh.normals.reshape(-1, 9),
                                  mesh.uvs.reshape(-1, 6)], axis=1).astype(np.float32)
            rec = np.zeros(mesh.triangle_count, [("f", "<f4", (24,)), ("m", "<u4")])
            rec["f"] = tri
            rec["m"] = mesh.material_ids
            rec.tofile(f)
            mesh.materials.tofile(f)
            textures.tofile(f)
            np.asarray(cam).tofile(f)
        r = subprocess.run([WRAPPER_BIN, scene, image], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        raw = np.fromfile(image, np.uint8)
    rgba_cxx = raw[:16 * w * h].view(np.float32).reshape(h, w, 4)
    counts_cxx = raw[16 * w * h:].view(np.uint32).reshape(h, w)
    params = default_params(background_r=0.1, background_g=0.1, background_b=0.1, max_path_depth=6,
                            min_samples=spp, max_samples_per_pixel=spp)
    tracer.configure(w, h, mesh)
    tracer.set_environment(None)
    tracer.set_camera(cam)
    tracer.set_params(params)
    tracer.reset_accumulation()
    tracer.render(0)
    rgba, counts, _ = tracer.readback()
    assert np.all(counts_cxx == spp) and np.array_equal(counts, counts_cxx)
    assert np.array_equal(rgba, rgba_cxx)
