"""B200 (sm_100a) path tracer standing in for LSystemEditor's PathTracerLib render path.

Public surface:
  * ``PathTracer``  -- host object over the C ABI in include/pt_b200.h
  * ``records``     -- byte layouts of materials, textures, camera, params
  * ``scene``       -- HostMesh container and the benchmark scene generator
"""
from .records import (CAMERA_DTYPE, MATERIAL_DTYPE, PARAMS_DTYPE, TEXTURE_DTYPE, default_material,  # noqa: F401
                      default_params, look_at_camera)
from .scene import HostMesh, SceneSpec, config0_scene  # noqa: F401


def __getattr__(name):
    if name in ("PathTracer", "PathTracerError", "load_library"):
        from . import pathtracer
        return getattr(pathtracer, name)
    raise AttributeError(name)
