"""Shared test helpers: seeded scenes and ray sets."""
import numpy as np

from lsystemeditor_b200.records import MATERIAL_DTYPE, TEXTURE_DTYPE, default_material, default_params, look_at_camera
from lsystemeditor_b200.scene import HostMesh, quad_mesh


def random_soup(n: int, seed: int = 0, extent: float = 4.0, size: float = 0.6, materials: int = 1) -> HostMesh:
    """Random triangles in a cube with random (unnormalised) vertex normals and uvs."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-extent, extent, (n, 1, 3))
    pos = (c + rng.normal(scale=size, size=(n, 3, 3))).astype(np.float32)
    face = np.cross(pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0])
    face /= np.linalg.norm(face, axis=1, keepdims=True) + 1e-12
    nrm = (face[:, None, :] + rng.normal(scale=0.2, size=(n, 3, 3))).astype(np.float32)
    uvs = rng.uniform(0, 1, (n, 3, 2)).astype(np.float32)
    mats = np.array([default_material(r=rng.uniform(0.1, 0.9), g=rng.uniform(0.1, 0.9), b=rng.uniform(0.1, 0.9),
                                      roughness=rng.uniform(0.05, 1.0)) for _ in range(materials)], MATERIAL_DTYPE)
    mids = rng.integers(0, materials, n).astype(np.uint32)
    return HostMesh(pos, nrm, uvs, mids, mats, np.zeros(0, TEXTURE_DTYPE))


def rays_through_bounds(mesh: HostMesh, n: int, seed: int = 1, pad: float = 1.0):
    rng = np.random.default_rng(seed)
    lo, hi = mesh.bounds()
    o = rng.uniform(lo - pad, hi + pad, (n, 3)).astype(np.float32)
    target = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = (target - o).astype(np.float32)
    return o, d


def material_zoo() -> np.ndarray:
    """One material per lobe combination the Principled BSDF distinguishes."""
    M = [
        default_material(r=0.7, g=0.6, b=0.5, roughness=0.6),                                   # diffuse+spec
        default_material(r=0.9, g=0.8, b=0.3, roughness=0.25, metallic=1.0),                    # metal
        default_material(r=0.95, g=0.95, b=0.95, roughness=0.02, transmission=1.0, ior=1.5),    # smooth glass
        default_material(r=0.9, g=0.9, b=0.95, roughness=0.4, transmission=1.0, ior=1.33),      # rough glass
        default_material(r=0.6, g=0.9, b=0.6, roughness=0.5, transmission=0.3, thin=1.0),       # thin leaf
        default_material(r=0.8, g=0.5, b=0.4, roughness=0.5, subsurface=1.0, scatter_radius_r=0.3,
                         scatter_radius_g=0.1, scatter_radius_b=0.05),                           # skin-like
        default_material(r=0.5, g=0.5, b=0.5, roughness=0.9, diffuse_roughness=0.2, specular=0.3),
        default_material(r=1.0, g=0.9, b=0.8, emission=4.0),                                    # emitter
    ]
    return np.array(M, MATERIAL_DTYPE)


def zoo_scene(n_per_mat: int = 300, seed: int = 3) -> HostMesh:
    soup = random_soup(n_per_mat * 8, seed=seed, extent=2.5, size=0.5, materials=8)
    soup.materials = material_zoo()
    tex = np.zeros(3, TEXTURE_DTYPE)
    tex[1]["kind"] = 2  # grid
    tex[1]["p0"] = [8.0, 8.0, 0.1, 0.0]
    tex[1]["p1"] = [0.1, 0.1, 0.1, 0.0]
    tex[1]["p2"] = [0.9, 0.9, 0.9, 0.0]
    tex[2]["kind"] = 3  # stripe, scalar
    tex[2]["p0"] = [6.0, 0.5, 0.9, 0.1]
    soup.materials[0]["albedo_tex"] = 1
    soup.materials[6]["roughness_tex"] = 2
    soup.textures = tex
    ground = quad_mesh((0, -3.2, 0), (12, 0, 0), (0, 0, -12), default_material(r=0.5, g=0.5, b=0.5, roughness=1.0),
                       normal=(0, 1, 0))
    light = quad_mesh((0, 4.0, 0), (2, 0, 0), (0, 0, 2), default_material(r=1, g=1, b=1, emission=8.0),
                      normal=(0, -1, 0))
    return HostMesh.concat([soup, ground, light])


def zoo_camera(w: int, h: int):
    return look_at_camera((0.5, 1.0, 9.0), (0.0, 0.0, 0.0), fov_y_deg=45.0, aspect=w / h)


def sky(width: int = 64, height: int = 32, seed: int = 5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    base = np.stack([0.3 + 0.7 * (1 - v), 0.4 + 0.5 * (1 - v), 0.8 + 0.2 * (1 - v)], -1)[:, None, :]
    img = np.broadcast_to(base, (height, width, 3)).copy()
    img[height // 5, width // 3] = [40.0, 38.0, 30.0]  # a sun
    img += rng.uniform(0, 0.05, img.shape)
    return img.astype(np.float32)


def rel_rmse(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-channel relative RMSE: sqrt(mean((a-b)^2)) / sqrt(mean(b^2))."""
    a = a.reshape(-1, a.shape[-1]).astype(np.float64)
    b = b.reshape(-1, b.shape[-1]).astype(np.float64)
    return np.sqrt(((a - b) ** 2).mean(0)) / np.maximum(np.sqrt((b ** 2).mean(0)), 1e-30)


def spectral_inputs(mesh: HostMesh, params, nw: int, env: np.ndarray = None) -> dict:
    """The spectral records the renderer derives from a scene (through its host functions), as the oracle's
    spectral render takes them: response table, per-material base / scatter coefficients, per-texture colour
    coefficients, per-texel environment coefficients, background x intensity."""
    from lsystemeditor_b200.pathtracer import PathTracer
    up = PathTracer.spectral_uplift
    m = mesh.materials if len(mesh.materials) else np.array([default_material()], MATERIAL_DTYPE)
    base = np.stack([m["r"], m["g"], m["b"]], 1)
    scat = np.stack([m["scatter_radius_r"], m["scatter_radius_g"], m["scatter_radius_b"]], 1)
    mat = np.concatenate([up(base), up(scat)], 1).astype(np.float32)
    tex = np.zeros((max(len(mesh.textures), 1), 8), np.float32)
    for i, t in enumerate(mesh.textures):
        if t["kind"] == 1:
            tex[i, :4] = up(t["p0"][:3])[0]
        elif t["kind"] == 2:
            tex[i, :4] = up(t["p1"][:3])[0]
            tex[i, 4:] = up(t["p2"][:3])[0]
    p = np.asarray(params).reshape(())
    k = np.float32(p["environment_intensity"])
    bg = up(np.array([p["background_r"] * k, p["background_g"] * k, p["background_b"] * k], np.float32))[0]
    envc = None if env is None else up(np.asarray(env, np.float32).reshape(-1, 3))
    return dict(nw=int(nw), resp=PathTracer.spectral_response(), mat=mat, tex=tex, env=envc, bg=bg)


def spectral_zoo_scene(n_per_mat: int = 300, seed: int = 3) -> HostMesh:
    """zoo_scene with coloured textures (a constant colour and a two-colour grid) and a tinted light."""
    mesh = zoo_scene(n_per_mat, seed)
    tex = np.zeros(4, TEXTURE_DTYPE)
    tex[:3] = mesh.textures[:3]
    tex[1]["p1"] = [0.8, 0.15, 0.1, 0.0]
    tex[1]["p2"] = [0.1, 0.3, 0.85, 0.0]
    tex[3]["kind"] = 1
    tex[3]["p0"] = [0.2, 0.7, 0.25, 0.0]
    mesh.textures = tex
    mesh.materials[6]["albedo_tex"] = 3
    mesh.materials[len(mesh.materials) - 1]["r"] = 1.0
    mesh.materials[len(mesh.materials) - 1]["g"] = 0.85
    mesh.materials[len(mesh.materials) - 1]["b"] = 0.6
    return mesh
