"""Python host API over the C ABI (include/pt_b200.h).

``PathTracer`` mirrors the reference renderer object
(PathTracerLib/src/PathTracer.h:30-152) minus Qt/OpenGL: configure, setters,
mesh rebuild, camera, render, headless readback, statistics and surface
picking.  Every call goes through ``libpt_b200.so``; there is no CPU fallback
-- construction fails if the library or a CUDA device is unavailable.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from . import _build
from .records import CAMERA_DTYPE, MATERIAL_DTYPE, PARAMS_DTYPE, TEXTURE_DTYPE
from .scene import HostMesh, TubeSet

PT_OK = 0
STATUS_NAMES = {0: "PT_OK", 1: "PT_ERR_INVALID_ARGUMENT", 2: "PT_ERR_CUDA", 3: "PT_ERR_OUT_OF_MEMORY",
                4: "PT_ERR_NO_SCENE", 5: "PT_ERR_NOT_CONFIGURED", 6: "PT_ERR_TIMEOUT", 7: "PT_ERR_UNSUPPORTED",
                8: "PT_ERR_INTERNAL"}

_fp = C.POINTER(C.c_float)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)


class PtMesh(C.Structure):
    _fields_ = [("triangle_count", C.c_uint32), ("positions", _fp), ("normals", _fp), ("uvs", _fp),
                ("material_ids", _u32p), ("material_count", C.c_uint32), ("materials", C.c_void_p),
                ("texture_count", C.c_uint32), ("textures", C.c_void_p)]


class PtTubes(C.Structure):
    _fields_ = [("tube_count", C.c_uint32), ("sides", C.c_uint32), ("ring_start", C.c_void_p),
                ("points", C.c_void_p), ("tangents", C.c_void_p), ("radii", C.c_void_p), ("materials", C.c_void_p),
                ("cos_sin", C.c_void_p), ("leaf_count", C.c_uint32), ("leaves", C.c_void_p),
                ("leaf_size", C.c_double), ("leaf_material", C.c_uint32), ("frames", C.c_void_p)]


class PtProfile(C.Structure):
    _fields_ = [("ms_generate", C.c_double), ("ms_extend", C.c_double), ("ms_shade", C.c_double),
                ("ms_shadow", C.c_double), ("ms_finalize", C.c_double), ("ms_accumulate", C.c_double),
                ("ms_compact", C.c_double), ("launches_extend", C.c_int64), ("launches_shadow", C.c_int64),
                ("rays_extend", C.c_int64), ("rays_shadow", C.c_int64), ("nodes_extend", C.c_int64),
                ("tris_extend", C.c_int64), ("nodes_shadow", C.c_int64), ("tris_shadow", C.c_int64)]


PROFILE_STAGE_TIMES = 1
PROFILE_COUNT_VISITS = 2


class PtInstance(C.Structure):
    _fields_ = [("object_to_world", C.c_float * 12), ("object", C.c_uint32), ("pad", C.c_uint32 * 3)]


class PtDistantLight(C.Structure):
    _fields_ = [("direction", C.c_float * 3), ("half_angle", C.c_float), ("radiance", C.c_float * 3),
                ("temperature_k", C.c_float), ("luminance", C.c_float), ("enabled", C.c_int32)]


class PtTuning(C.Structure):
    _fields_ = [("path_capacity", C.c_int32), ("blocks_per_sm", C.c_int32), ("samples_per_launch", C.c_int32),
                ("trials", C.c_int32), ("ms_default", C.c_double), ("ms_best", C.c_double)]


class PtStats(C.Structure):
    _fields_ = [("waves", C.c_int64), ("active_pixels", C.c_int64), ("samples", C.c_int64), ("rays", C.c_int64),
                ("launches", C.c_int64), ("render_ms", C.c_double), ("build_ms", C.c_double),
                ("budget_exhausted", C.c_int32), ("bvh_nodes", C.c_int32), ("tape_underruns", C.c_int32),
                ("stack_overflows", C.c_int32)]


EXPORTED_SYMBOLS = ["pt_create", "pt_destroy", "pt_last_error", "pt_configure", "pt_set_mesh", "pt_set_camera",
                    "pt_get_camera", "pt_set_params", "pt_get_params", "pt_default_params", "pt_set_environment",
                    "pt_reset", "pt_render", "pt_readback", "pt_device_buffers", "pt_get_stats", "pt_trace_rays",
                    "pt_trace_rays_device", "pt_rng_tape", "pt_set_stream", "pt_set_profiling", "pt_get_profile",
                    "pt_set_tuning", "pt_trace_soup_noalloc", "pt_batch_configure", "pt_batch_set_mesh",
                    "pt_batch_set_camera", "pt_batch_readback", "pt_batch_set_tubes", "pt_export_mesh",
                    "pt_tonemap", "pt_exposure_multiplier", "pt_set_materials", "pt_backward",
                    "pt_record_samples", "pt_set_preview_levels", "pt_render_previews", "pt_preview_readback", "pt_set_region",
                    "pt_reset_region", "pt_environment_tables", "pt_spectral_response", "pt_spectral_uplift",
                    "pt_set_instances", "pt_set_distant_light", "pt_batch_share_scene", "pt_autotune", "pt_measure_l2",
                    "pt_set_extend_mode", "pt_radix_sort_temp_bytes", "pt_radix_sort_pairs",
                    "pt_set_bvh_options", "pt_bvh_sah_cost"]

_LIB: Optional[C.CDLL] = None


def load_library(build_if_missing: bool = True) -> C.CDLL:
    """Loads libpt_b200.so (building it with nvcc first when it is missing or stale)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB
    if build_if_missing and _build.needs_build():
        _build.build()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing; run lsystemeditor_b200._build.build()")
    L = C.CDLL(path)
    vp = C.c_void_p
    L.pt_create.argtypes = [C.POINTER(vp), C.c_int]
    L.pt_destroy.argtypes = [vp]
    L.pt_last_error.argtypes = [vp]
    L.pt_last_error.restype = C.c_char_p
    L.pt_configure.argtypes = [vp, C.c_int, C.c_int]
    L.pt_set_mesh.argtypes = [vp, C.POINTER(PtMesh)]
    L.pt_set_camera.argtypes = [vp, vp]
    L.pt_get_camera.argtypes = [vp, vp]
    L.pt_set_params.argtypes = [vp, vp]
    L.pt_get_params.argtypes = [vp, vp]
    L.pt_default_params.argtypes = [vp]
    L.pt_default_params.restype = None
    L.pt_set_environment.argtypes = [vp, C.c_int, C.c_int, _fp]
    L.pt_reset.argtypes = [vp]
    L.pt_render.argtypes = [vp, C.c_int]
    L.pt_readback.argtypes = [vp, _fp, _u32p, _u8p]
    L.pt_device_buffers.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    L.pt_get_stats.argtypes = [vp, C.POINTER(PtStats)]
    L.pt_trace_rays.argtypes = [vp, C.c_int, _fp, _fp, _fp, _fp, _u8p, _fp, _u32p, _fp, _fp]
    L.pt_trace_rays_device.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.pt_rng_tape.argtypes = [vp, C.c_int, C.c_int, C.c_int, _fp]
    L.pt_set_stream.argtypes = [vp, vp]
    L.pt_set_profiling.argtypes = [vp, C.c_int]
    L.pt_get_profile.argtypes = [vp, C.POINTER(PtProfile)]
    L.pt_set_tuning.argtypes = [vp, C.c_int, C.c_int]
    L.pt_set_extend_mode.argtypes = [vp, C.c_int]
    L.pt_batch_configure.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pt_batch_set_mesh.argtypes = [vp, C.c_int, C.POINTER(PtMesh)]
    L.pt_batch_set_camera.argtypes = [vp, C.c_int, vp]
    L.pt_batch_readback.argtypes = [vp, C.c_int, _fp, _u32p, _u8p]
    L.pt_batch_set_tubes.argtypes = [vp, C.c_int, C.POINTER(PtTubes), C.POINTER(PtMesh)]
    L.pt_export_mesh.argtypes = [vp, C.c_int, _u32p, _fp, _fp, _fp, _u32p]
    L.pt_tonemap.argtypes = [vp, C.c_int, C.c_float, _u8p]
    L.pt_exposure_multiplier.argtypes = [C.c_float, C.c_float, C.c_float]
    L.pt_exposure_multiplier.restype = C.c_float
    L.pt_set_materials.argtypes = [vp, C.c_int, C.c_uint32, vp]
    L.pt_backward.argtypes = [vp, _fp, C.c_int, C.c_int, _fp, C.c_uint32, C.POINTER(C.c_double)]
    L.pt_record_samples.argtypes = [vp, C.c_int]
    L.pt_set_preview_levels.argtypes = [vp, C.c_int]
    L.pt_render_previews.argtypes = [vp]
    L.pt_preview_readback.argtypes = [vp, C.c_int, _fp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pt_set_region.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L.pt_reset_region.argtypes = [vp]
    L.pt_environment_tables.argtypes = [vp, _fp, _fp]
    L.pt_spectral_response.argtypes = [_fp, _fp, _fp]
    L.pt_spectral_uplift.argtypes = [C.c_uint32, _fp, _fp]
    L.pt_set_instances.argtypes = [vp, C.c_int, C.c_uint32, C.POINTER(PtMesh), C.c_uint32, C.POINTER(PtInstance)]
    L.pt_set_distant_light.argtypes = [vp, C.POINTER(PtDistantLight)]
    L.pt_batch_share_scene.argtypes = [vp, C.c_int, C.c_int]
    L.pt_autotune.argtypes = [vp, C.c_int, C.POINTER(PtTuning)]
    L.pt_measure_l2.argtypes = [vp, C.c_uint64, C.c_int, C.POINTER(C.c_double)]
    L.pt_set_bvh_options.argtypes = [vp, C.c_int]
    L.pt_bvh_sah_cost.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
    L.pt_radix_sort_temp_bytes.argtypes = [C.c_uint32]
    L.pt_radix_sort_temp_bytes.restype = C.c_size_t
    L.pt_radix_sort_pairs.argtypes = [vp, vp, vp, vp, C.c_uint32, C.c_int, vp, C.c_size_t, vp]
    _LIB = L
    return L


class PathTracerError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


class PathTracer:
    """Renderer object (reference: class PathTracer, PathTracer.h:30-152)."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        h = C.c_void_p()
        rc = self._lib.pt_create(C.byref(h), int(device))
        if rc != PT_OK:
            raise PathTracerError(rc, "pt_create failed (is a CUDA device available?)")
        self._h = h
        self._mesh_keepalive = None
        self.width = 0
        self.height = 0
        self._params = np.zeros((), PARAMS_DTYPE)
        self._lib.pt_default_params(C.c_void_p(self._params.ctypes.data))

    # -- lifetime -------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.pt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != PT_OK:
            msg = self._lib.pt_last_error(self._h)
            raise PathTracerError(rc, msg.decode() if msg else "")

    # -- configure / scene ------------------------------------------------
    def configure(self, width: int, height: int, mesh: Optional[HostMesh] = None):
        """PathTracer::configure (PathTracer.h:45-51) without GL surfaces."""
        self._check(self._lib.pt_configure(self._h, int(width), int(height)))
        self.width, self.height = int(width), int(height)
        self.batch_sizes = [(self.width, self.height)]
        if mesh is not None:
            self.set_mesh(mesh)

    @staticmethod
    def _pt_mesh(mesh: HostMesh):
        m = mesh.contiguous()
        s = PtMesh(m.triangle_count, _ptr(m.positions, _fp), _ptr(m.normals, _fp), _ptr(m.uvs, _fp),
                   _ptr(m.material_ids, _u32p), len(m.materials),
                   C.c_void_p(m.materials.ctypes.data) if len(m.materials) else None, len(m.textures),
                   C.c_void_p(m.textures.ctypes.data) if len(m.textures) else None)
        return m, s

    def set_mesh(self, mesh: HostMesh):
        """MeshAccelScene::build + upload / PathTracer::rebuildMeshScene: GPU BVH build."""
        m, s = self._pt_mesh(mesh)
        self._check(self._lib.pt_set_mesh(self._h, C.byref(s)))
        self._mesh_keepalive = m

    rebuild_mesh_scene = set_mesh

    def set_instances(self, objects, instances, scene: int = 0):
        """Instanced scene: `objects` (list of HostMesh; objects[0]'s material and texture banks serve all) placed
        by `instances`, a list of (object_to_world 3x4, object index).  One BVH per object, a top-level BVH over
        the instances, both built on the device."""
        keep = [self._pt_mesh(m) for m in objects]
        arr = (PtMesh * len(keep))(*[s for _, s in keep])
        inst = (PtInstance * len(instances))()
        for k, (mat, obj) in enumerate(instances):
            m = np.asarray(mat, np.float32).reshape(3, 4)
            inst[k].object_to_world = (C.c_float * 12)(*m.reshape(-1).tolist())
            inst[k].object = int(obj)
        self._check(self._lib.pt_set_instances(self._h, int(scene), len(keep), arr, len(instances), inst))
        self._mesh_keepalive = [m for m, _ in keep]

    def set_distant_light(self, direction=None, half_angle: float = 0.0, radiance=(0.0, 0.0, 0.0),
                          temperature_k: float = 0.0, luminance: float = 1.0):
        """Distant light in a cone of `half_angle` radians around `direction` (towards the light): RGB
        `radiance`, or a blackbody of `temperature_k` with Rec. 709 luminance `luminance`.  None removes it."""
        if direction is None:
            self._check(self._lib.pt_set_distant_light(self._h, None))
            return
        l = PtDistantLight()
        l.direction = (C.c_float * 3)(*[float(x) for x in direction])
        l.half_angle = float(half_angle)
        l.radiance = (C.c_float * 3)(*[float(x) for x in radiance])
        l.temperature_k = float(temperature_k)
        l.luminance = float(luminance)
        l.enabled = 1
        self._check(self._lib.pt_set_distant_light(self._h, C.byref(l)))

    def set_camera(self, camera: np.ndarray):
        cam = np.ascontiguousarray(camera, CAMERA_DTYPE)
        self._check(self._lib.pt_set_camera(self._h, C.c_void_p(cam.ctypes.data)))

    def last_sample_camera(self) -> np.ndarray:
        cam = np.zeros((), CAMERA_DTYPE)
        self._check(self._lib.pt_get_camera(self._h, C.c_void_p(cam.ctypes.data)))
        return cam

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, PARAMS_DTYPE)
        self._check(self._lib.pt_set_params(self._h, C.c_void_p(p.ctypes.data)))
        self._params = p.copy()

    def params(self) -> np.ndarray:
        p = np.zeros((), PARAMS_DTYPE)
        self._check(self._lib.pt_get_params(self._h, C.c_void_p(p.ctypes.data)))
        return p

    def _set(self, **kw):
        p = self.params()
        for k, v in kw.items():
            p[k] = v
        self.set_params(p)

    # Setters of the reference (PathTracer.h:73-124); values are clamped the
    # way PathTracer.cpp:126-190 clamps them.
    def set_max_samples_per_pixel(self, n: int):
        self._set(max_samples_per_pixel=int(min(max(n, 0), 1_000_000)))

    def set_min_samples(self, n: int):
        self._set(min_samples=int(min(max(n, 1), 10_000)))

    def set_relative_error_threshold(self, t: float):
        self._set(relative_error_threshold=float(min(max(t, 0.001), 1.0)))

    def set_russian_roulette_min_depth(self, d: int):
        self._set(russian_roulette_min_depth=int(max(d, 0)))

    def set_brdf_debug_flags(self, flags: int):
        self._set(brdf_debug_flags=int(flags))

    def set_debug_overlay_mode(self, mode: int):
        self._set(debug_overlay_mode=int(mode))

    def set_clear_color(self, r: float, g: float, b: float):
        self._set(background_r=r, background_g=g, background_b=b)

    def set_environment_intensity(self, k: float):
        self._set(environment_intensity=float(k))

    def set_max_path_depth(self, d: int):
        self._set(max_path_depth=int(d))

    def set_environment(self, rgb: Optional[np.ndarray]):
        """Lat-long linear RGB (H, W, 3) or None for the solid background."""
        if rgb is None:
            self._check(self._lib.pt_set_environment(self._h, 0, 0, None))
            return
        a = np.ascontiguousarray(rgb, np.float32)
        self._check(self._lib.pt_set_environment(self._h, a.shape[1], a.shape[0], _ptr(a, _fp)))

    # -- rendering --------------------------------------------------------
    def environment_tables(self, width: int, height: int):
        """The environment map's marginal and row CDFs as built on the device."""
        marg = np.empty(height + 1, np.float32)
        row = np.empty((height, width + 1), np.float32)
        self._check(self._lib.pt_environment_tables(self._h, _ptr(marg, _fp), _ptr(row, _fp)))
        return marg, row

    def reset_accumulation(self):
        self._check(self._lib.pt_reset(self._h))

    def render(self, waves: int = 0):
        """Traces `waves` full-resolution adaptive waves (<= 0: until every pixel is done)."""
        self._check(self._lib.pt_render(self._h, int(waves)))

    def readback(self, out: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None
                 ) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """pt_readback: accumulated RGBA, sample counts and convergence flags of scene 0.  `out` reuses
        caller-owned arrays (e.g. pinned host memory) of shapes (H, W, 4) float32, (H, W) uint32, (H, W) uint8."""
        P = self.width * self.height
        if out is None:
            rgba = np.empty((self.height, self.width, 4), np.float32)
            counts = np.empty((self.height, self.width), np.uint32)
            conv = np.empty((self.height, self.width), np.uint8)
        else:
            rgba, counts, conv = out
            ok = (rgba.dtype == np.float32 and rgba.size == 4 * P and counts.dtype == np.uint32 and counts.size == P
                  and conv.dtype == np.uint8 and conv.size == P and all(a.flags["C_CONTIGUOUS"] for a in out))
            if not ok:
                raise ValueError("readback: out arrays must be C-contiguous float32 (H, W, 4), uint32 and uint8 (H, W)")
        self._check(self._lib.pt_readback(self._h, _ptr(rgba, _fp), _ptr(counts, _u32p), _ptr(conv, _u8p)))
        assert rgba.size == 4 * P
        return rgba, counts, conv

    def device_buffers(self) -> Tuple[int, int, int]:
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._check(self._lib.pt_device_buffers(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def stats(self) -> dict:
        s = PtStats()
        self._check(self._lib.pt_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in PtStats._fields_}

    def current_sample_count(self) -> int:
        return int(self.stats()["waves"])

    def current_active_pixel_count(self) -> int:
        return int(self.stats()["active_pixels"])

    def is_sample_budget_exhausted(self) -> bool:
        return bool(self.stats()["budget_exhausted"])

    def sample_budget_total_iterations(self) -> int:
        """PathTracerSampleBudget.h:8-14 with no preview levels."""
        m = int(self.params()["max_samples_per_pixel"])
        return -1 if m <= 0 else m

    # -- batched form (no reference counterpart) -------------------------------
    def batch_configure(self, sizes):
        """Several independent scenes rendered together; sizes = [(width, height), ...].
        The single-scene calls then address scene 0."""
        w = (C.c_int * len(sizes))(*[int(a) for a, _ in sizes])
        h = (C.c_int * len(sizes))(*[int(b) for _, b in sizes])
        self._check(self._lib.pt_batch_configure(self._h, len(sizes), w, h))
        self.batch_sizes = [(int(a), int(b)) for a, b in sizes]
        self.width, self.height = self.batch_sizes[0]

    def batch_set_mesh(self, scene: int, mesh: HostMesh):
        m, s = self._pt_mesh(mesh)
        self._check(self._lib.pt_batch_set_mesh(self._h, int(scene), C.byref(s)))

    def batch_share_scene(self, scene: int, source: int):
        """Scene `scene` renders scene `source`'s geometry with its own camera and image (one BVH, several views)."""
        self._check(self._lib.pt_batch_share_scene(self._h, int(scene), int(source)))

    def batch_set_camera(self, scene: int, camera: np.ndarray):
        cam = np.ascontiguousarray(camera, CAMERA_DTYPE)
        self._check(self._lib.pt_batch_set_camera(self._h, int(scene), C.c_void_p(cam.ctypes.data)))

    def batch_readback(self, scene: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        w, h = self.batch_sizes[scene]
        rgba = np.empty((h, w, 4), np.float32)
        counts = np.empty((h, w), np.uint32)
        conv = np.empty((h, w), np.uint8)
        self._check(self._lib.pt_batch_readback(self._h, int(scene), _ptr(rgba, _fp), _ptr(counts, _u32p),
                                                _ptr(conv, _u8p)))
        return rgba, counts, conv

    # -- scene generation on the device, export, display --------------------
    def set_procedural(self, instances, params=None, scene: int = 0):
        """meshSceneBuild (MeshSceneContent.h:16-20) over ProceduralInstance records: the
        instances' turtle output in world space (procedural.build_tubes) lofted and built
        on the device into scene `scene` (pt_batch_set_tubes).  Returns the TubeSet."""
        from .procedural import build_tubes
        tubes = build_tubes(instances, params)
        self.batch_set_tubes(scene, tubes)
        return tubes

    def batch_set_tubes(self, scene: int, tubes: TubeSet):
        """Lofts tubes and leaves on the GPU (pt_batch_set_tubes) and builds scene `scene`."""
        rs = np.ascontiguousarray(tubes.ring_start, np.uint32)
        pts = np.ascontiguousarray(tubes.points, np.float64)
        tan = np.ascontiguousarray(tubes.tangents, np.float64)
        rad = np.ascontiguousarray(tubes.radii, np.float64)
        mat = np.ascontiguousarray(tubes.materials, np.uint32)
        cs = np.ascontiguousarray(tubes.cos_sin(), np.float64)
        lv = np.ascontiguousarray(tubes.leaves, np.float64)
        addr = lambda a: C.c_void_p(a.ctypes.data) if a.size else None
        fr = None if tubes.frames is None else np.ascontiguousarray(tubes.frames, np.float64)
        t = PtTubes(len(mat), int(tubes.sides), addr(rs), addr(pts), addr(tan), addr(rad), addr(mat), addr(cs),
                    len(lv), addr(lv), float(tubes.leaf_size), int(tubes.leaf_material),
                    addr(fr) if fr is not None else None)
        m, ms = self._pt_mesh(tubes.extra)
        self._check(self._lib.pt_batch_set_tubes(self._h, int(scene), C.byref(t), C.byref(ms)))

    def export_mesh(self, scene: int = 0) -> HostMesh:
        """The scene's triangles as built on the device (original order); material bank not included."""
        n = C.c_uint32()
        self._check(self._lib.pt_export_mesh(self._h, int(scene), C.byref(n), None, None, None, None))
        N = int(n.value)
        pos = np.empty((N, 3, 3), np.float32); nrm = np.empty((N, 3, 3), np.float32)
        uv = np.empty((N, 3, 2), np.float32); mid = np.empty(N, np.uint32)
        if N:
            self._check(self._lib.pt_export_mesh(self._h, int(scene), C.byref(n), _ptr(pos, _fp), _ptr(nrm, _fp),
                                                 _ptr(uv, _fp), _ptr(mid, _u32p)))
        from .records import MATERIAL_DTYPE as _M, TEXTURE_DTYPE as _T
        return HostMesh(pos, nrm, uv, mid, np.zeros(0, _M), np.zeros(0, _T))

    def tonemap(self, scene: int = 0, exposure: float = 1.0) -> np.ndarray:
        """8-bit RGBA display image (reference display pipeline), (height, width, 4) uint8."""
        w, h = (self.batch_sizes[scene] if getattr(self, "batch_sizes", None) and scene > 0
                else (self.width, self.height))
        out = np.empty((h, w, 4), np.uint8)
        self._check(self._lib.pt_tonemap(self._h, int(scene), float(exposure), _ptr(out, _u8p)))
        return out

    @staticmethod
    def exposure_multiplier(f_stop: float, shutter_seconds: float, iso: float) -> float:
        """PhysicalCamera::exposureMultiplier (PhysicalCamera.cpp:392-397)."""
        return float(load_library().pt_exposure_multiplier(float(f_stop), float(shutter_seconds), float(iso)))

    # -- spectral mode (params["spectral_wavelengths"] = 4 or 8) --------------
    @staticmethod
    def spectral_response() -> np.ndarray:
        """sRGB response per nm, 380 .. 780 nm (401 x 3); each channel sums to 1 (trapezoid rule)."""
        out = np.empty((401, 3), np.float32)
        rc = load_library().pt_spectral_response(_ptr(out, _fp), None, None)
        if rc != PT_OK:
            raise PathTracerError(rc, "pt_spectral_response failed")
        return out

    @staticmethod
    def spectral_source_tables() -> Tuple[np.ndarray, np.ndarray]:
        """(x-bar, y-bar, z-bar, D65) at 380 .. 780 nm every 10 nm (41 x 4) and the XYZ -> sRGB matrix."""
        cie = np.empty((41, 4), np.float32)
        m = np.empty((3, 3), np.float32)
        rc = load_library().pt_spectral_response(None, _ptr(cie, _fp), _ptr(m, _fp))
        if rc != PT_OK:
            raise PathTracerError(rc, "pt_spectral_response failed")
        return cie, m

    @staticmethod
    def spectral_uplift(rgb) -> np.ndarray:
        """Spectrum coefficients (c0, c1, c2, scale), lambda in nm, of RGB colours (n x 3) as the renderer uses
        them: scale * (1/2 + x / (2 sqrt(1 + x^2))), x = c0 lambda^2 + c1 lambda + c2."""
        a = np.ascontiguousarray(np.asarray(rgb, np.float32).reshape(-1, 3))
        out = np.empty((len(a), 4), np.float32)
        rc = load_library().pt_spectral_uplift(len(a), _ptr(a, _fp), _ptr(out, _fp))
        if rc != PT_OK:
            raise PathTracerError(rc, "pt_spectral_uplift failed")
        return out

    # -- preview passes and region render (PathTracer.h:89-92, 134-140) --------
    def set_preview_steps_per_level(self, levels: int):
        """PathTracer::setPreviewStepsPerLevel: low-resolution preview passes before full resolution."""
        self._check(self._lib.pt_set_preview_levels(self._h, int(levels)))

    def render_previews(self):
        """Renders the preview passes (pt_render does it before its first wave anyway)."""
        self._check(self._lib.pt_render_previews(self._h))

    def preview(self, level: int) -> np.ndarray:
        w, h = C.c_int(), C.c_int()
        self._check(self._lib.pt_preview_readback(self._h, int(level), None, C.byref(w), C.byref(h)))
        out = np.empty((h.value, w.value, 4), np.float32)
        self._check(self._lib.pt_preview_readback(self._h, int(level), _ptr(out, _fp), C.byref(w), C.byref(h)))
        return out

    def set_render_region(self, min_x: int, min_y: int, max_x: int, max_y: int, enabled: bool = True):
        """setRegionRenderEnabled + setRenderRegion: only the rectangle takes samples."""
        self._check(self._lib.pt_set_region(self._h, int(bool(enabled)), int(min_x), int(min_y), int(max_x),
                                            int(max_y)))

    def reset_region_accumulation(self):
        self._check(self._lib.pt_reset_region(self._h))

    # -- differentiation (no reference counterpart) -----------------------------
    GRAD_PARAMS = ("r", "g", "b", "roughness", "metallic", "sheen", "emission")

    def set_materials(self, materials: np.ndarray, scene: int = 0):
        """Replaces the material bank (same ids) without rebuilding the BVH."""
        m = np.ascontiguousarray(materials, MATERIAL_DTYPE)
        self._check(self._lib.pt_set_materials(self._h, int(scene), len(m), C.c_void_p(m.ctypes.data)))

    def record_samples(self, spp: int):
        """Keep every sample's radiance of fixed-spp renders for backward (0 = off)."""
        self._check(self._lib.pt_record_samples(self._h, int(spp)))

    def backward(self, d_image: np.ndarray, spp: int, materials: int = 16):
        """Path-replay gradient of a loss through the image pt_render draws with
        `spp` samples per pixel: d_image is d loss / d image (H, W, 3 or 4).
        Returns (grad (materials, 7) in GRAD_PARAMS order, device milliseconds)."""
        d = np.ascontiguousarray(d_image, np.float32)
        ch = d.shape[-1]
        assert d.size == self.width * self.height * ch and ch in (3, 4)
        g = np.zeros((materials, 7), np.float32)
        ms = C.c_double()
        self._check(self._lib.pt_backward(self._h, _ptr(d, _fp), int(ch), int(spp), _ptr(g, _fp), int(materials),
                                          C.byref(ms)))
        return g, float(ms.value)

    # -- queries ----------------------------------------------------------
    def trace_rays(self, origins, dirs, tmin=None, tmax=None) -> dict:
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        n = o.shape[0]
        tmin = np.zeros(n, np.float32) if tmin is None else np.ascontiguousarray(np.broadcast_to(tmin, (n,)), np.float32)
        tmax = np.full(n, 1.0e6, np.float32) if tmax is None else np.ascontiguousarray(np.broadcast_to(tmax, (n,)), np.float32)
        hit = np.zeros(n, np.uint8); t = np.zeros(n, np.float32); tri = np.zeros(n, np.uint32)
        nrm = np.zeros((n, 3), np.float32); uv = np.zeros((n, 2), np.float32)
        self._check(self._lib.pt_trace_rays(self._h, n, _ptr(o, _fp), _ptr(d, _fp), _ptr(tmin, _fp), _ptr(tmax, _fp),
                                            _ptr(hit, _u8p), _ptr(t, _fp), _ptr(tri, _u32p), _ptr(nrm, _fp),
                                            _ptr(uv, _fp)))
        return dict(hit=hit.astype(bool), t=t, tri=tri, normal=nrm, uv=uv)

    def pick_surface(self, origin, direction):
        """PathTracer::pickSurface (PathTracer.cpp:1991-2013): tMin 0.001, tMax 1e30."""
        r = self.trace_rays(np.asarray(origin)[None], np.asarray(direction)[None], 0.001, 1.0e30)
        return {k: v[0] for k, v in r.items()}

    def autotune(self, waves: int = 8) -> dict:
        """pt_autotune: path capacity, blocks per SM and waves per launch chosen by timing `waves`-wave renders of
        the current setup (the image does not depend on them); the accumulation is reset afterwards."""
        t = PtTuning()
        self._check(self._lib.pt_autotune(self._h, int(waves), C.byref(t)))
        self._params["samples_per_launch"] = t.samples_per_launch
        return {f: getattr(t, f) for f, _ in PtTuning._fields_}

    def measure_l2(self, nbytes: int = 32 << 20, reps: int = 64) -> float:
        """pt_measure_l2: L2-resident read bandwidth in GB/s."""
        v = C.c_double()
        self._check(self._lib.pt_measure_l2(self._h, int(nbytes), int(reps), C.byref(v)))
        return float(v.value)

    # -- runtime plumbing ---------------------------------------------------
    def set_stream(self, stream_handle: Optional[int]):
        """Issue all work on a caller's CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self._lib.pt_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def set_profiling(self, flags: int):
        self._check(self._lib.pt_set_profiling(self._h, int(flags)))

    def profile(self) -> dict:
        p = PtProfile()
        self._check(self._lib.pt_get_profile(self._h, C.byref(p)))
        return {k: getattr(p, k) for k, _ in PtProfile._fields_}

    def set_tuning(self, path_capacity: int = 0, blocks_per_sm: int = 0):
        self._check(self._lib.pt_set_tuning(self._h, int(path_capacity), int(blocks_per_sm)))

    def set_bvh_options(self, treelet_passes: int = 1):
        """Treelet SAH reordering passes of the next BVH builds (0 = plain Karras LBVH)."""
        self._check(self._lib.pt_set_bvh_options(self._h, int(treelet_passes)))

    def bvh_sah_cost(self, scene: int = 0) -> float:
        c = C.c_double()
        self._check(self._lib.pt_bvh_sah_cost(self._h, int(scene), C.byref(c)))
        return float(c.value)

    def set_extend_mode(self, mode: int):
        """pt_set_extend_mode: 0 auto, 1 warp-fetch closest hit, 2 per-lane replacement (identical images)."""
        self._check(self._lib.pt_set_extend_mode(self._h, int(mode)))

    def rng_tape(self, first_wave: int, waves: int, stride: int) -> np.ndarray:
        out = np.zeros((waves, self.width * self.height, stride), np.float32)
        self._check(self._lib.pt_rng_tape(self._h, int(first_wave), int(waves), int(stride), _ptr(out, _fp)))
        return out
