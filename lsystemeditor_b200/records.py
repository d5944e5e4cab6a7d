"""Byte layouts shared by the C ABI (include/pt_b200.h) and the Python host code.

Each record keeps the field order and size of the reference struct it stands
in for, so that a caller holding the reference's structs can pass them through
unchanged:

==================  =====  ==============================================================
record              bytes  reference struct
==================  =====  ==============================================================
MATERIAL_DTYPE        96   ``MaterialGpu``      PathTracerLib/src/MeshAccel/MeshAccelTypes.h:49-86
TEXTURE_DTYPE         64   ``TextureDescGpu``   PathTracerLib/src/MeshAccel/MeshAccelTypes.h:22-28
CAMERA_DTYPE          80   ``CameraGpu``        PathTracerLib/src/CameraGpu.h:5-16
PARAMS_DTYPE          80   ``RenderParamsGpu``  PathTracerLib/src/RenderTypes.h:15-28 (44 B) + extensions
==================  =====  ==============================================================

``MATERIAL_DTYPE`` uses the reference's 4 tail-padding bytes for ``sheen``
(no counterpart in the reference; 0 disables it).  ``PARAMS_DTYPE`` appends
fields after the reference's 44 bytes; a zero-filled tail selects the
reference behaviour.
"""
from __future__ import annotations

import numpy as np

MATERIAL_DTYPE = np.dtype([
    ("r", "<f4"), ("g", "<f4"), ("b", "<f4"),
    ("roughness", "<f4"), ("metallic", "<f4"), ("transmission", "<f4"),
    ("thin", "<f4"), ("ior", "<f4"), ("subsurface", "<f4"), ("emission", "<f4"),
    ("diffuse_roughness", "<f4"),
    ("scatter_radius_r", "<f4"), ("scatter_radius_g", "<f4"), ("scatter_radius_b", "<f4"),
    ("specular", "<f4"),
    ("albedo_tex", "<u4"), ("roughness_tex", "<u4"), ("metallic_tex", "<u4"),
    ("transmission_tex", "<u4"), ("thin_tex", "<u4"), ("ior_tex", "<u4"),
    ("subsurface_tex", "<u4"), ("emission_tex", "<u4"),
    ("sheen", "<f4"),
])
assert MATERIAL_DTYPE.itemsize == 96

TEXTURE_DTYPE = np.dtype([
    ("kind", "<u4"), ("pad", "<u4", (3,)),
    ("p0", "<f4", (4,)), ("p1", "<f4", (4,)), ("p2", "<f4", (4,)),
])
assert TEXTURE_DTYPE.itemsize == 64

# TextureKind (MeshAccelTypes.h:13-19).
TEX_CONSTANT_SCALAR, TEX_CONSTANT_RGB, TEX_GRID_2D, TEX_STRIPE_1D = 0, 1, 2, 3

CAMERA_DTYPE = np.dtype([
    ("position", "<f4", (3,)), ("pad0", "<f4"),
    ("orientation", "<f4", (4,)),  # quaternion (w, x, y, z)
    ("fov_y", "<f4"), ("aspect", "<f4"), ("near_plane", "<f4"), ("far_plane", "<f4"),
    ("aperture_radius", "<f4"), ("focus_distance", "<f4"),
    ("focus_point", "<f4", (3,)), ("focus_valid", "<i4"), ("pad1", "<f4", (2,)),
])
assert CAMERA_DTYPE.itemsize == 80

PARAMS_DTYPE = np.dtype([
    # --- RenderParamsGpu (44 bytes) ---
    ("background_r", "<f4"), ("background_g", "<f4"), ("background_b", "<f4"),
    ("environment_intensity", "<f4"),
    ("max_path_depth", "<i4"), ("russian_roulette_min_depth", "<i4"),
    ("min_samples", "<i4"), ("max_samples_per_pixel", "<i4"),
    ("debug_overlay_mode", "<i4"), ("brdf_debug_flags", "<i4"),
    ("relative_error_threshold", "<f4"),
    # --- extensions (zero = reference behaviour) ---
    ("seed_mode", "<i4"),            # 0: reference seed formula, 1: hash(x, y, seed_value)
    ("seed_value", "<u4"),
    ("adaptive_criterion", "<i4"),   # 0: relative std-dev (reference), 1: relative std-error, 2: as 1 + black stops
    ("samples_per_launch", "<i4"),   # 0: automatic batch of waves per launch
    ("spectral_wavelengths", "<i4"), # 0: RGB (reference); 4 or 8 hero wavelengths
    ("emitter_mis", "<i4"),          # 0: reference emissive NEE; 1: MIS-complete emitters at opaque vertices
    ("reserved", "<i4", (3,)),
])
assert PARAMS_DTYPE.itemsize == 80

REFERENCE_PARAMS_BYTES = 44


def default_material(**kw) -> np.ndarray:
    """``MaterialGpu{}`` defaults (MeshAccelTypes.h:49-86) with keyword overrides."""
    m = np.zeros((), MATERIAL_DTYPE)
    m["r"] = m["g"] = m["b"] = 0.8
    m["roughness"] = 0.5
    m["ior"] = 1.5
    m["diffuse_roughness"] = -1.0
    m["specular"] = 1.0
    for k, v in kw.items():
        m[k] = v
    return m


def default_params(**kw) -> np.ndarray:
    """``RenderParamsGpu{}`` defaults (RenderTypes.h:15-28) with keyword overrides."""
    p = np.zeros((), PARAMS_DTYPE)
    p["background_r"] = p["background_g"] = p["background_b"] = np.float32(10.0) / np.float32(255.0)
    p["environment_intensity"] = 1.0
    p["max_path_depth"] = 32
    p["russian_roulette_min_depth"] = 3
    p["min_samples"] = 16
    p["max_samples_per_pixel"] = 1024
    p["relative_error_threshold"] = 0.02
    for k, v in kw.items():
        p[k] = v
    return p


def quat_from_basis(right, up, back) -> np.ndarray:
    """Unit quaternion (w, x, y, z) of the rotation whose columns are right, up, back."""
    m = np.stack([right, up, back], axis=1).astype(np.float64)
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    if tr > 0:
        s = np.sqrt(tr + 1.0) * 2
        w, x, y, z = 0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s
    elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = np.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2
        w, x, y, z = (m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s
    elif m[1, 1] > m[2, 2]:
        s = np.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2
        w, x, y, z = (m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s
    else:
        s = np.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2
        w, x, y, z = (m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s
    q = np.array([w, x, y, z])
    return (q / np.linalg.norm(q)).astype(np.float32)


def look_at_camera(eye, target, up=(0.0, 1.0, 0.0), fov_y_deg=40.0, aspect=1.0,
                   near=0.1, far=1000.0, aperture_radius=0.0, focus_distance=0.0) -> np.ndarray:
    """Pinhole (``focus_valid = 0``) or thin-lens camera record looking from eye to target.

    The camera looks down its local -Z axis with +Y up (CameraDevice.cuh:8-50).
    """
    eye = np.asarray(eye, np.float64)
    target = np.asarray(target, np.float64)
    fwd = target - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    c = np.zeros((), CAMERA_DTYPE)
    c["position"] = eye
    c["orientation"] = quat_from_basis(right, upv, -fwd)
    c["fov_y"] = np.deg2rad(fov_y_deg)
    c["aspect"] = aspect
    c["near_plane"] = near
    c["far_plane"] = far
    c["aperture_radius"] = aperture_radius
    c["focus_distance"] = focus_distance
    c["focus_point"] = eye + fwd * focus_distance
    c["focus_valid"] = 1 if (aperture_radius > 0 and focus_distance > 0) else 0
    return c
