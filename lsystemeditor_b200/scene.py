"""Host-side mesh container and the procedural scene generator for the benchmark scenes.

``HostMesh`` is the flat structure-of-arrays form of the reference's
``HostMesh`` (Application/src/MeshBuilder/HostMesh.h:9-28): per triangle three
positions, three shading normals, three uvs and a material index, plus the
material and texture banks.

The generator is a small L-system rewriter + turtle + tube loft that produces
the benchmark scenes.  It follows the reference's turtle conventions
(Application/src/Procedural/Turtle.cpp:12-282): the turtle starts at the
origin heading -Z with up +Y, ``Yaw`` turns about up, ``Pitch`` about
right = up x tangent, ``Roll`` about the tangent, ``F`` appends a state and
brackets / ``f`` close the current segment.  Each segment is lofted as an
n-gon tube with rings at its states and flat caps (Loft.cpp:108-155).  It is a
scene generator only; the path tracer consumes whatever mesh it is given.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .records import MATERIAL_DTYPE, TEXTURE_DTYPE, default_material, default_params, look_at_camera


@dataclasses.dataclass
class HostMesh:
    positions: np.ndarray        # (N, 3, 3) float32
    normals: np.ndarray          # (N, 3, 3) float32
    uvs: np.ndarray              # (N, 3, 2) float32
    material_ids: np.ndarray     # (N,) uint32
    materials: np.ndarray        # (M,) MATERIAL_DTYPE
    textures: np.ndarray         # (K,) TEXTURE_DTYPE

    @property
    def triangle_count(self) -> int:
        return int(self.positions.shape[0])

    @staticmethod
    def empty() -> "HostMesh":
        return HostMesh(np.zeros((0, 3, 3), np.float32), np.zeros((0, 3, 3), np.float32),
                        np.zeros((0, 3, 2), np.float32), np.zeros((0,), np.uint32),
                        np.zeros((0,), MATERIAL_DTYPE), np.zeros((0,), TEXTURE_DTYPE))

    def contiguous(self) -> "HostMesh":
        return HostMesh(np.ascontiguousarray(self.positions, np.float32),
                        np.ascontiguousarray(self.normals, np.float32),
                        np.ascontiguousarray(self.uvs, np.float32),
                        np.ascontiguousarray(self.material_ids, np.uint32),
                        np.ascontiguousarray(self.materials, MATERIAL_DTYPE),
                        np.ascontiguousarray(self.textures, TEXTURE_DTYPE))

    @staticmethod
    def concat(parts: Sequence["HostMesh"]) -> "HostMesh":
        """Appends meshes like hostMeshAppend (HostMesh.h:77-117): material ids are offset."""
        pos, nrm, uv, mid, mats, texs = [], [], [], [], [], []
        mat_off = 0
        for p in parts:
            pos.append(p.positions)
            nrm.append(p.normals)
            uv.append(p.uvs)
            mid.append(p.material_ids.astype(np.uint32) + np.uint32(mat_off))
            mats.append(p.materials)
            texs.append(p.textures)
            mat_off += len(p.materials)
        return HostMesh(np.concatenate(pos).astype(np.float32), np.concatenate(nrm).astype(np.float32),
                        np.concatenate(uv).astype(np.float32), np.concatenate(mid).astype(np.uint32),
                        np.concatenate(mats), np.concatenate(texs))

    def bounds(self) -> Tuple[np.ndarray, np.ndarray]:
        p = self.positions.reshape(-1, 3)
        return p.min(axis=0), p.max(axis=0)


def quad_mesh(center, u_axis, v_axis, material: np.ndarray, normal=None) -> HostMesh:
    """Two-triangle rectangle spanning center +- u_axis/2 +- v_axis/2."""
    c = np.asarray(center, np.float32)
    u = np.asarray(u_axis, np.float32) * 0.5
    v = np.asarray(v_axis, np.float32) * 0.5
    p00, p10, p11, p01 = c - u - v, c + u - v, c + u + v, c - u + v
    n = np.cross(u, v) if normal is None else np.asarray(normal, np.float32)
    n = (n / np.linalg.norm(n)).astype(np.float32)
    pos = np.array([[p00, p10, p11], [p00, p11, p01]], np.float32)
    nrm = np.broadcast_to(n, (2, 3, 3)).astype(np.float32)
    uvs = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], np.float32)
    return HostMesh(pos, nrm, uvs, np.zeros(2, np.uint32), np.atleast_1d(material).astype(MATERIAL_DTYPE),
                    np.zeros(0, TEXTURE_DTYPE))


# ---------------------------------------------------------------------------
# L-system rewriting.  A module is (name, args); rules map a name to a
# function of (args, rng) returning the successor module list.
# ---------------------------------------------------------------------------
Module = Tuple[str, Tuple[float, ...]]
Rule = Callable[[Tuple[float, ...], np.random.Generator], List[Module]]


def expand(axiom: List[Module], rules: Dict[str, Rule], iterations: int, seed: int = 0) -> List[Module]:
    rng = np.random.default_rng(seed)
    word = list(axiom)
    for _ in range(iterations):
        out: List[Module] = []
        for name, args in word:
            rule = rules.get(name)
            if rule is None:
                out.append((name, args))
            else:
                out.extend(rule(args, rng))
        word = out
    return word


# ---------------------------------------------------------------------------
# Turtle (Turtle.cpp:110-282).
# ---------------------------------------------------------------------------
def _rotate(v: np.ndarray, axis: np.ndarray, deg: float) -> np.ndarray:
    n = axis / np.linalg.norm(axis)
    a = math.radians(deg)
    c, s = math.cos(a), math.sin(a)
    return v * c + np.cross(n, v) * s + n * np.dot(n, v) * (1.0 - c)


@dataclasses.dataclass
class Segment:
    points: List[np.ndarray]
    tangents: List[np.ndarray]
    radii: List[float]
    material: int
    tag: int  # caller-defined (branch depth for leaves, etc.)


def turtle(word: List[Module], start_tangent=(0.0, 0.0, -1.0), start_up=(0.0, 1.0, 0.0),
           default_step: float = 1.0, default_radius: float = 0.1,
           leaf_symbol: Optional[str] = None) -> Tuple[List[Segment], List[Tuple[np.ndarray, np.ndarray, np.ndarray, float]]]:
    """Runs the turtle; returns tube segments and leaf frames (position, tangent, up, size)."""
    pos = np.zeros(3)
    tan = np.asarray(start_tangent, np.float64)
    up = np.asarray(start_up, np.float64)
    stack: List[Tuple[np.ndarray, np.ndarray, np.ndarray, int]] = []
    states: List[Tuple[np.ndarray, np.ndarray, float]] = []
    segments: List[Segment] = []
    leaves: List[Tuple[np.ndarray, np.ndarray, np.ndarray, float]] = []
    material = 0

    def flush():
        nonlocal states
        if not states:
            return
        last_r = states[-1][2]
        states.append((pos.copy(), tan.copy(), last_r))
        segments.append(Segment([s[0] for s in states], [s[1] for s in states], [s[2] for s in states],
                                material, len(stack)))
        states = []

    for name, args in word:
        if name == "[":
            flush()
            stack.append((pos.copy(), tan.copy(), up.copy(), material))
        elif name == "]":
            flush()
            if stack:
                pos, tan, up, material = stack.pop()
        elif name == "F":
            step = args[0] if args else default_step
            radius = args[1] if len(args) > 1 else (args[0] if args else default_radius)
            states.append((pos.copy(), tan.copy(), float(radius)))
            pos = pos + tan * step
        elif name == "f":
            flush()
            pos = pos + tan * (args[0] if args else default_step)
        elif name == "Yaw":
            tan = _rotate(tan, up, args[0]); up = _rotate(up, up, args[0])
            tan /= np.linalg.norm(tan); up /= np.linalg.norm(up)
        elif name in ("Pitch", "Pich"):
            right = np.cross(up, tan); right /= np.linalg.norm(right)
            tan = _rotate(tan, right, args[0]); up = _rotate(up, right, args[0])
            tan /= np.linalg.norm(tan); up /= np.linalg.norm(up)
        elif name == "Roll":
            up = _rotate(up, tan, args[0]); up /= np.linalg.norm(up)
        elif name == "Mat":
            material = int(args[0])
        elif leaf_symbol is not None and name == leaf_symbol:
            leaves.append((pos.copy(), tan.copy(), up.copy(), float(args[0]) if args else 1.0))
    flush()
    return segments, leaves


# ---------------------------------------------------------------------------
# Loft (Loft.cpp:108-155): rings at every state, side quads as two triangles,
# flat caps at both ends.  Vectorised over all segments that have the same
# number of rings.
# ---------------------------------------------------------------------------
def _perp_frames(tangents: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    t = tangents / np.linalg.norm(tangents, axis=-1, keepdims=True)
    ref = np.where(np.abs(t[..., 1:2]) < 0.99, np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    a = np.cross(ref, t)
    a /= np.linalg.norm(a, axis=-1, keepdims=True)
    b = np.cross(t, a)
    return a, b


def loft(segments: Sequence[Segment], sides: int = 8, material_ids: Optional[Sequence[int]] = None) -> HostMesh:
    groups: Dict[int, List[int]] = {}
    for i, s in enumerate(segments):
        groups.setdefault(len(s.points), []).append(i)
    parts_pos, parts_nrm, parts_uv, parts_mid = [], [], [], []
    ang = np.arange(sides + 1) * (2.0 * math.pi / sides)
    cs, sn = np.cos(ang), np.sin(ang)
    for rings, idxs in groups.items():
        P = np.array([[segments[i].points[k] for k in range(rings)] for i in idxs])      # (S, R, 3)
        T = np.array([[segments[i].tangents[k] for k in range(rings)] for i in idxs])
        Rr = np.array([[segments[i].radii[k] for k in range(rings)] for i in idxs])     # (S, R)
        T[:, -1] = T[:, -2] if rings > 1 else T[:, -1]
        A, B = _perp_frames(T)
        # Parallel-transport-free approximation: per-ring frame from the ring tangent.
        dirs = A[:, :, None, :] * cs[None, None, :, None] + B[:, :, None, :] * sn[None, None, :, None]  # (S,R,C+1,3)
        ringp = P[:, :, None, :] + dirs * Rr[:, :, None, None]
        S = len(idxs)
        tris_pos, tris_nrm, tris_uv = [], [], []
        for r in range(rings - 1):
            v0, v1 = r / max(rings - 1, 1), (r + 1) / max(rings - 1, 1)
            for k in range(sides):
                a00, a01 = ringp[:, r, k], ringp[:, r, k + 1]
                a10, a11 = ringp[:, r + 1, k], ringp[:, r + 1, k + 1]
                n00, n01 = dirs[:, r, k], dirs[:, r, k + 1]
                n10, n11 = dirs[:, r + 1, k], dirs[:, r + 1, k + 1]
                u0, u1 = k / sides, (k + 1) / sides
                tris_pos += [np.stack([a00, a01, a10], 1), np.stack([a01, a11, a10], 1)]
                tris_nrm += [np.stack([n00, n01, n10], 1), np.stack([n01, n11, n10], 1)]
                uvq = np.array([[[u0, v0], [u1, v0], [u0, v1]], [[u1, v0], [u1, v1], [u0, v1]]], np.float32)
                tris_uv += [np.broadcast_to(uvq[0], (S, 3, 2)), np.broadcast_to(uvq[1], (S, 3, 2))]
        # caps
        for end, sign in ((0, -1.0), (rings - 1, 1.0)):
            tn = T[:, end] / np.linalg.norm(T[:, end], axis=-1, keepdims=True) * sign
            c = P[:, end]
            for k in range(sides):
                r0, r1 = ringp[:, end, k], ringp[:, end, k + 1]
                tri = np.stack([c, r1, r0] if sign < 0 else [c, r0, r1], 1)
                tris_pos.append(tri)
                tris_nrm.append(np.broadcast_to(tn[:, None, :], (S, 3, 3)))
                tris_uv.append(np.broadcast_to(np.array([[0.5, 0.5], [1.0, 0.0], [0.0, 1.0]], np.float32), (S, 3, 2)))
        pos = np.stack(tris_pos, 1).reshape(-1, 3, 3)     # segment-major
        nrm = np.stack(tris_nrm, 1).reshape(-1, 3, 3)
        uv = np.stack(tris_uv, 1).reshape(-1, 3, 2)
        per = len(tris_pos)
        mids = np.repeat(np.array([segments[i].material if material_ids is None else material_ids[i]
                                   for i in idxs], np.uint32), per)
        parts_pos.append(pos); parts_nrm.append(nrm); parts_uv.append(uv); parts_mid.append(mids)
    if not parts_pos:
        return HostMesh.empty()
    return HostMesh(np.concatenate(parts_pos).astype(np.float32), np.concatenate(parts_nrm).astype(np.float32),
                    np.concatenate(parts_uv).astype(np.float32), np.concatenate(parts_mid).astype(np.uint32),
                    np.zeros(0, MATERIAL_DTYPE), np.zeros(0, TEXTURE_DTYPE))


def leaf_quads(leaves, size: float, material: int) -> HostMesh:
    """One two-triangle quad per leaf frame, spanning the leaf's up/tangent plane."""
    if not leaves:
        return HostMesh.empty()
    P = np.array([l[0] for l in leaves]); T = np.array([l[1] for l in leaves]); U = np.array([l[2] for l in leaves])
    s = np.array([l[3] for l in leaves])[:, None] * size
    w = np.cross(T, U)
    w /= np.linalg.norm(w, axis=-1, keepdims=True)
    p00, p10 = P - w * s * 0.5, P + w * s * 0.5
    p01, p11 = p00 + T * s, p10 + T * s
    n = U / np.linalg.norm(U, axis=-1, keepdims=True)
    pos = np.stack([np.stack([p00, p10, p11], 1), np.stack([p00, p11, p01], 1)], 1).reshape(-1, 3, 3)
    nrm = np.repeat(n[:, None, None, :], 2, 1).repeat(3, 2).reshape(-1, 3, 3)
    uv1 = np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], np.float32)
    uvs = np.broadcast_to(uv1, (len(leaves), 2, 3, 2)).reshape(-1, 3, 2)
    return HostMesh(pos.astype(np.float32), nrm.astype(np.float32), uvs.astype(np.float32),
                    np.full(len(leaves) * 2, material, np.uint32), np.zeros(0, MATERIAL_DTYPE),
                    np.zeros(0, TEXTURE_DTYPE))


# ---------------------------------------------------------------------------
# Tube sets: turtle output in the form the device loft takes (pt_tubes).
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class TubeSet:
    """Branch tubes + leaf frames + extra triangles, lofted on the GPU by
    pt_batch_set_tubes; ``host_mesh`` is the same loft on the host (the
    device result is bit-identical when every tube has the same ring count)."""
    ring_start: np.ndarray   # (T + 1,) uint32
    points: np.ndarray       # (R, 3) float64 ring centres
    tangents: np.ndarray     # (R, 3) float64
    radii: np.ndarray        # (R,) float64
    materials: np.ndarray    # (T,) uint32, index into extra.materials
    sides: int
    leaves: np.ndarray       # (L, 10) float64: position, tangent, up, size
    leaf_size: float
    leaf_material: int
    extra: HostMesh          # appended triangles; its material bank is the scene's

    @staticmethod
    def from_turtle(segments: Sequence[Segment], leaves, sides: int, leaf_size: float, leaf_material: int,
                    extra: HostMesh, tube_material_offset: int = 0) -> "TubeSet":
        counts = np.array([len(sg.points) for sg in segments], np.int64)
        ring_start = np.zeros(len(segments) + 1, np.uint32)
        ring_start[1:] = np.cumsum(counts)
        if segments:
            pts = np.array([p for sg in segments for p in sg.points], np.float64).reshape(-1, 3)
            tans = np.array([t for sg in segments for t in sg.tangents], np.float64).reshape(-1, 3)
            rad = np.array([r for sg in segments for r in sg.radii], np.float64)
        else:
            pts = np.zeros((0, 3)); tans = np.zeros((0, 3)); rad = np.zeros(0)
        mats = np.array([sg.material + tube_material_offset for sg in segments], np.uint32)
        lv = np.array([np.concatenate([l[0], l[1], l[2], [l[3]]]) for l in leaves], np.float64).reshape(-1, 10)
        return TubeSet(ring_start, pts, tans, rad, mats, int(sides), lv, float(leaf_size), int(leaf_material),
                       extra)

    @property
    def triangle_count(self) -> int:
        return 2 * self.sides * len(self.radii) + 2 * len(self.leaves) + self.extra.triangle_count

    def cos_sin(self) -> np.ndarray:
        """The loft's angle table (same expression as ``loft``)."""
        ang = np.arange(self.sides + 1) * (2.0 * math.pi / self.sides)
        return np.stack([np.cos(ang), np.sin(ang)], -1).reshape(-1)

    def segments(self) -> List[Segment]:
        out = []
        for t in range(len(self.materials)):
            a, b = int(self.ring_start[t]), int(self.ring_start[t + 1])
            out.append(Segment(list(self.points[a:b]), list(self.tangents[a:b]), list(self.radii[a:b]),
                               int(self.materials[t]), 0))
        return out

    def host_mesh(self) -> HostMesh:
        """The same mesh built on the host: tubes, leaves, extra."""
        segs = self.segments()
        tube = loft(segs, self.sides, material_ids=[int(m) for m in self.materials]) if segs else HostMesh.empty()
        lv = [(r[0:3], r[3:6], r[6:9], float(r[9])) for r in self.leaves]
        leaf = leaf_quads(lv, self.leaf_size, self.leaf_material)
        parts = [tube, leaf, self.extra]
        return HostMesh(np.concatenate([q.positions for q in parts]).astype(np.float32),
                        np.concatenate([q.normals for q in parts]).astype(np.float32),
                        np.concatenate([q.uvs for q in parts]).astype(np.float32),
                        np.concatenate([q.material_ids for q in parts]).astype(np.uint32),
                        self.extra.materials, self.extra.textures)

    def bounds(self) -> Tuple[np.ndarray, np.ndarray]:
        """Bounds of the ring centres padded by the radii and of the leaf bases (a conservative estimate)."""
        lo = np.full(3, np.inf); hi = np.full(3, -np.inf)
        if len(self.radii):
            lo = np.minimum(lo, (self.points - self.radii[:, None]).min(0))
            hi = np.maximum(hi, (self.points + self.radii[:, None]).max(0))
        if len(self.leaves):
            lo = np.minimum(lo, self.leaves[:, 0:3].min(0) - self.leaf_size)
            hi = np.maximum(hi, self.leaves[:, 0:3].max(0) + self.leaf_size)
        return lo, hi


# ---------------------------------------------------------------------------
# Benchmark scenes.
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class SceneSpec:
    name: str
    mesh: HostMesh
    camera: np.ndarray
    params: np.ndarray
    width: int
    height: int
    waves: int  # number of full-resolution waves a complete render takes (upper bound)
    tubes: Optional["TubeSet"] = None  # the same scene as tubes + leaves + extra triangles (device loft)


def bracketed_ol_tree(iterations: int = 4, angle: float = 25.7, length: float = 0.1, radius: float = 0.02,
                      sides: int = 8) -> HostMesh:
    """F(h,r) -> F(h,r)[Yaw(a)F(h,r)]F(h,r)[Yaw(-a)F(h,r)]F(h,r) in the XY plane (5^n segments).

    The turtle heads +Y with up +Z so that Yaw bends the branches in the XY plane
    (the reference reaches the same orientation with a +90 degree instance pitch).
    """
    def rule(args, _rng):
        h, r = args
        F = ("F", (h, r))
        return [F, ("[", ()), ("Yaw", (angle,)), F, ("]", ()), F, ("[", ()), ("Yaw", (-angle,)), F, ("]", ()), F]
    word = expand([("F", (length, radius))], {"F": rule}, iterations)
    segs, _ = turtle(word, start_tangent=(0.0, 1.0, 0.0), start_up=(0.0, 0.0, 1.0))
    return loft(segs, sides)


def stochastic_tree(iterations: int = 7, seed: int = 7, angle: float = 22.5, jitter: float = 5.0,
                    length: float = 0.8, radius: float = 0.08, length_decay: float = 0.9, radius_decay: float = 0.7):
    """3D stochastic L-system tree: axiom A,
        A -> F [&+A] [&-A] [^A]   (p = 0.6)
        A -> F [&A] [^/A]         (p = 0.4)
    with + / - = Yaw(+-a), & / ^ = Pitch(+-a), / = Roll(a), a = angle +- uniform jitter
    (drawn per symbol from a seeded generator and baked into the successor), segment
    length x length_decay and radius x radius_decay per depth.  Terminal A's carry
    a leaf.  Returns (segments, leaves) from the turtle (heading +Y, up +Z).
    """
    def rot(name, rng, sign=1.0):
        return (name, (sign * (angle + rng.uniform(-jitter, jitter)),))

    def rule(args, rng):
        depth = args[0]
        h = length * length_decay ** depth
        r = radius * radius_decay ** depth
        F = ("F", (h, r))
        A = ("A", (depth + 1,))
        if rng.uniform() < 0.6:
            return [F, ("[", ()), rot("Pitch", rng), rot("Yaw", rng), A, ("]", ()),
                    ("[", ()), rot("Pitch", rng), rot("Yaw", rng, -1.0), A, ("]", ()),
                    ("[", ()), rot("Pitch", rng, -1.0), A, ("]", ())]
        return [F, ("[", ()), rot("Pitch", rng), A, ("]", ()),
                ("[", ()), rot("Pitch", rng, -1.0), rot("Roll", rng), A, ("]", ())]

    word = expand([("A", (0,))], {"A": rule}, iterations, seed=seed)
    word = [("Leaf", (1.0,)) if name == "A" else (name, a) for name, a in word]
    return turtle(word, start_tangent=(0.0, 1.0, 0.0), start_up=(0.0, 0.0, 1.0), leaf_symbol="Leaf")


def refine_segments(segments: Sequence[Segment], rings: int, taper: float) -> List[Segment]:
    """Resamples every two-state segment into `rings` states with a linear radius taper."""
    out = []
    for s in segments:
        p0, p1 = s.points[0], s.points[-1]
        r0 = s.radii[0]
        pts = [p0 + (p1 - p0) * (k / (rings - 1)) for k in range(rings)]
        tans = [s.tangents[0]] * rings
        radii = [r0 * (1.0 - (1.0 - taper) * k / (rings - 1)) for k in range(rings)]
        out.append(Segment(pts, tans, radii, s.material, s.tag))
    return out


def _bank(materials) -> HostMesh:
    """A mesh without triangles that carries a material bank (for HostMesh.concat)."""
    e = HostMesh.empty()
    e.materials = np.array(list(materials), MATERIAL_DTYPE)
    return e


BARK = dict(r=0.35, g=0.22, b=0.12, roughness=0.8)
LEAF = dict(r=0.1, g=0.4, b=0.08, roughness=0.5, transmission=0.3, thin=1.0)


def tree_tubes(iterations: int = 7, seed: int = 7, sides: int = 64, rings: int = 16, taper: float = 0.85,
               leaf_size: float = 0.18) -> TubeSet:
    """The stochastic tree as a TubeSet: bark tubes (material 0), leaf quads
    (material 1), the ground (2) and the light (3) of the plain scenes."""
    segs, leaves = stochastic_tree(iterations=iterations, seed=seed)
    segs = refine_segments(segs, rings, taper=taper)
    ground = quad_mesh((0, 0, 0), (10, 0, 0), (0, 0, -10),
                       default_material(r=0.5, g=0.5, b=0.5, roughness=1.0), normal=(0, 1, 0))
    light = quad_mesh((0, 5, 1.5), (1, 0, 0), (0, 0, 1),
                      default_material(r=1.0, g=1.0, b=1.0, emission=10.0), normal=(0, -1, 0))
    extra = HostMesh.concat([_bank([default_material(**BARK), default_material(**LEAF)]), ground, light])
    return TubeSet.from_turtle(segs, leaves, sides, leaf_size, leaf_material=1, extra=extra)


def config1_scene(width: int = 1024, height: int = 1024, sides: int = 64, rings: int = 16,
                  max_depth: int = 12) -> SceneSpec:
    """Plain method, large: the 3D stochastic tree (7 iterations, seed 7) with leaf quads.

    The grammar yields ~500 branch segments and ~800 leaves; to reach the ~1M
    triangles of the workload each branch is lofted as a 64-gon tube with 16
    tapered rings.  Bark (0.35, 0.22, 0.12) roughness 0.8; leaves (0.1, 0.4,
    0.08) roughness 0.5, transmission 0.3, thin; the light and ground of the
    plain-small scene.  1024^2, adaptive 16..1024 spp stopping at a relative
    standard error of 1e-2, max depth 12.  ``tubes`` holds the same scene for
    the device loft.
    """
    tubes = tree_tubes(sides=sides, rings=rings)
    mesh = tubes.host_mesh()
    n_tree = 2 * tubes.sides * len(tubes.radii) + 2 * len(tubes.leaves)
    p = mesh.positions[:n_tree].reshape(-1, 3)
    lo, hi = p.min(axis=0), p.max(axis=0)
    center = (lo + hi) * 0.5
    extent = float(np.max(hi - lo))
    dist = extent * 0.5 / math.tan(math.radians(20.0)) * 1.2
    cam = look_at_camera((center[0], center[1], center[2] + dist), center, fov_y_deg=40.0, aspect=width / height)
    params = default_params(background_r=0.0, background_g=0.0, background_b=0.0, max_path_depth=max_depth,
                            russian_roulette_min_depth=3, min_samples=16, max_samples_per_pixel=1024,
                            relative_error_threshold=0.01, adaptive_criterion=1)
    spec = SceneSpec(f"plain-large: 3D stochastic L-system tree, {mesh.triangle_count} triangles, 1024x1024, "
                     "adaptive 16-1024 spp to relative std-error 1e-2, depth 12", mesh, cam, params, width, height,
                     1024)
    spec.tubes = tubes
    return spec


def batch_scenes(count: int = 64, seed: int = 2, sides: int = 48, rings: int = 16, max_depth: int = 12,
                 min_spp: int = 16, max_spp: int = 512, rel_err: float = 0.03):
    """Batching workload: `count` stochastic trees of the plain-large grammar with
    iterations drawn uniformly from 4..8, L-system seeds 100, 101, ..., image
    sizes drawn from 256^2, 512^2, 768^2, 1024^2 and cameras orbiting the tree
    at a seeded azimuth (every draw from numpy's default generator seeded with
    `seed`).  Tubes are 48-gons with 16 rings (about 40M triangles over 64
    scenes).  Shared params: adaptive min_spp..max_spp stopping at a relative
    standard error of `rel_err` (0.03, i.e. a per-pixel relative MSE of about
    1e-3), depth 12, black background.  Returns (tubes, cameras, sizes, params).
    """
    rng = np.random.default_rng(seed)
    its = rng.integers(4, 9, count)
    res = rng.choice(np.array([256, 512, 768, 1024]), count)
    az = rng.uniform(0.0, 2.0 * math.pi, count)
    tubes, cams, sizes = [], [], []
    for k in range(count):
        t = tree_tubes(iterations=int(its[k]), seed=100 + k, sides=sides, rings=rings)
        lo, hi = t.bounds()
        center = (lo + hi) * 0.5
        extent = float(np.max(hi - lo))
        dist = extent * 0.5 / math.tan(math.radians(20.0)) * 1.2
        eye = (center[0] + dist * math.sin(az[k]), center[1] + 0.15 * dist, center[2] + dist * math.cos(az[k]))
        w = h = int(res[k])
        tubes.append(t)
        cams.append(look_at_camera(eye, center, fov_y_deg=40.0, aspect=w / h))
        sizes.append((w, h))
    params = default_params(background_r=0.0, background_g=0.0, background_b=0.0, max_path_depth=max_depth,
                            russian_roulette_min_depth=3, min_samples=min_spp, max_samples_per_pixel=max_spp,
                            relative_error_threshold=rel_err, adaptive_criterion=1)
    return tubes, cams, sizes, params


def diff_materials(rng: np.random.Generator, count: int = 8) -> np.ndarray:
    """Seeded Principled parameters of the differentiation workload: base colour
    in U[0.05, 0.9]^3, roughness in U[0.1, 1], metallic in U[0, 0.3], sheen in
    U[0, 0.5] (sheen is this project's extension lobe)."""
    mats = []
    for _ in range(count):
        c = rng.uniform(0.05, 0.9, 3)
        mats.append(default_material(r=c[0], g=c[1], b=c[2], roughness=rng.uniform(0.1, 1.0),
                                     metallic=rng.uniform(0.0, 0.3), sheen=rng.uniform(0.0, 0.5)))
    return np.array(mats, MATERIAL_DTYPE)


def config3_scene(width: int = 512, height: int = 512, spp: int = 64, seed: int = 3, max_depth: int = 8) -> SceneSpec:
    """Differentiation: the plain-small geometry with 8 branch materials chosen by
    depth along the tree (8 equal bands of the distance of a segment's start from
    the root), the ground (material 8) and the light (material 9, emission
    strength in U[5, 20]); seeded ground-truth parameters (diff_materials);
    fixed `spp`, max depth 8, black background."""
    def rule(args, _rng):
        h, r = args
        F = ("F", (h, r))
        a = 25.7
        return [F, ("[", ()), ("Yaw", (a,)), F, ("]", ()), F, ("[", ()), ("Yaw", (-a,)), F, ("]", ()), F]
    word = expand([("F", (0.1, 0.02))], {"F": rule}, 4)
    segs, _ = turtle(word, start_tangent=(0.0, 1.0, 0.0), start_up=(0.0, 0.0, 1.0))
    dist = np.array([float(np.linalg.norm(sg.points[0])) for sg in segs])
    band = np.minimum((dist / max(dist.max(), 1e-9) * 8.0).astype(int), 7)
    tree = loft(segs, 8, material_ids=[int(b) for b in band])
    rng = np.random.default_rng(seed)
    tree.materials = diff_materials(rng, 8)
    ground = quad_mesh((0, 0, 0), (10, 0, 0), (0, 0, -10),
                       default_material(r=0.5, g=0.5, b=0.5, roughness=1.0), normal=(0, 1, 0))
    light = quad_mesh((0, 5, 1.5), (1, 0, 0), (0, 0, 1),
                      default_material(r=1.0, g=1.0, b=1.0, emission=rng.uniform(5.0, 20.0)), normal=(0, -1, 0))
    mesh = HostMesh.concat([tree, ground, light])
    lo, hi = tree.bounds()
    center = (lo + hi) * 0.5
    extent = float(np.max(hi - lo))
    dist_c = extent * 0.5 / math.tan(math.radians(20.0)) * 1.15
    cam = look_at_camera((center[0], center[1], center[2] + dist_c), center, fov_y_deg=40.0, aspect=width / height)
    params = default_params(background_r=0.0, background_g=0.0, background_b=0.0, max_path_depth=max_depth,
                            russian_roulette_min_depth=3, min_samples=spp, max_samples_per_pixel=spp)
    return SceneSpec(f"differentiation: bracketed tree with 8 depth materials, {width}x{height}, {spp} spp",
                     mesh, cam, params, width, height, spp)


def config0_scene(width: int = 256, height: int = 256, spp: int = 64, max_depth: int = 8) -> SceneSpec:
    """Plain method, small: 625-segment bracketed tree, ground, one area light, pinhole 40 deg.

    Bark (0.35, 0.22, 0.12) roughness 0.8; ground 0.5 grey roughness 1; a 1x1
    light at height 5 (emission 10, white) offset 1.5 units in z so that the trunk
    does not pass through it; black background; 64 spp fixed (min = max); max depth 8.
    """
    tree = bracketed_ol_tree()
    tree.materials = np.array([default_material(r=0.35, g=0.22, b=0.12, roughness=0.8, metallic=0.0)],
                              MATERIAL_DTYPE)
    ground = quad_mesh((0, 0, 0), (10, 0, 0), (0, 0, -10),
                       default_material(r=0.5, g=0.5, b=0.5, roughness=1.0), normal=(0, 1, 0))
    light = quad_mesh((0, 5, 1.5), (1, 0, 0), (0, 0, 1),
                      default_material(r=1.0, g=1.0, b=1.0, emission=10.0), normal=(0, -1, 0))
    mesh = HostMesh.concat([tree, ground, light])
    lo, hi = tree.bounds()
    center = (lo + hi) * 0.5
    extent = float(np.max(hi - lo))
    dist = extent * 0.5 / math.tan(math.radians(20.0)) * 1.15
    cam = look_at_camera((center[0], center[1], center[2] + dist), center, fov_y_deg=40.0,
                         aspect=width / height)
    params = default_params(background_r=0.0, background_g=0.0, background_b=0.0, max_path_depth=max_depth,
                            russian_roulette_min_depth=3, min_samples=spp, max_samples_per_pixel=spp)
    return SceneSpec("plain-small: 2D bracketed OL-system, 625 segments, 256x256, 64 spp, depth 8",
                     mesh, cam, params, width, height, spp)


@dataclasses.dataclass
class InstancedScene:
    """Objects placed by instances (pt_set_instances).  ``objects[0]``'s material
    and texture banks serve every object.  ``flatten`` bakes the instances into
    one mesh, which is what the reference does with its ProceduralInstance list
    (MeshSceneContent.h:16-20): the instanced render is checked against it."""
    objects: List[HostMesh]
    instances: List[Tuple[np.ndarray, int]]   # (3x4 object-to-world, object index)

    @property
    def triangle_count(self) -> int:
        return int(sum(self.objects[o].triangle_count for _, o in self.instances))

    @property
    def unique_triangles(self) -> int:
        return int(sum(m.triangle_count for m in self.objects))

    def flatten(self) -> HostMesh:
        parts = []
        for mat, o in self.instances:
            m = self.objects[o]
            M = np.asarray(mat, np.float64).reshape(3, 4)
            A, t = M[:, :3], M[:, 3]
            N = np.linalg.inv(A).T
            pos = (m.positions.reshape(-1, 3).astype(np.float64) @ A.T + t).astype(np.float32)
            nrm = (m.normals.reshape(-1, 3).astype(np.float64) @ N.T).astype(np.float32)
            parts.append(HostMesh(pos.reshape(-1, 3, 3), nrm.reshape(-1, 3, 3), m.uvs, m.material_ids,
                                  np.zeros((0,), MATERIAL_DTYPE), np.zeros((0,), TEXTURE_DTYPE)))
        flat = HostMesh.concat(parts)
        flat.materials = self.objects[0].materials
        flat.textures = self.objects[0].textures
        return flat


def placement(x: float, z: float, yaw: float, scale: float, y: float = 0.0) -> np.ndarray:
    """3x4 object-to-world matrix: uniform scale, rotation about +Y by yaw (radians), translation."""
    c, s = math.cos(yaw), math.sin(yaw)
    return np.array([[scale * c, 0.0, scale * s, x], [0.0, scale, 0.0, y], [-scale * s, 0.0, scale * c, z]],
                    np.float32)


SUN_TEMPERATURE = 5800.0
SUN_HALF_ANGLE = math.radians(0.53) * 0.5


def forest_scene(width: int = 1920, height: int = 1080, trees: int = 12, instances: int = 500, seed: int = 200,
                 extent: float = 200.0, sides: int = 40, rings: int = 16, views: int = 4, max_depth: int = 16,
                 min_spp: int = 32, max_spp: int = 2048, rel_err: float = 0.01, iterations=(6, 8)):
    """Large instanced forest: `trees` distinct stochastic trees of the plain-large
    grammar (iterations drawn from 6..8, L-system seeds seed .. seed + trees - 1),
    `instances` placements at seeded positions on an extent x extent ground with
    random yaw and scale 0.7..1.3, the ground as one more object.  Light: a
    sun-like distant light (0.53 degree cone, 5800 K blackbody, elevation 35
    degrees) plus a uniform sky.  Cameras: `views` views orbiting the centre at
    a seeded azimuth (the batched form renders them in one launch).  Adaptive
    min_spp..max_spp to a relative standard error of rel_err, depth 16.  The
    small forms used by the tests shrink `iterations`, `extent` and the counts.

    Returns (InstancedScene, cameras, params, sun) with sun = dict(direction,
    half_angle, temperature_k, luminance)."""
    rng = np.random.default_rng(seed)
    its = rng.integers(iterations[0], iterations[1] + 1, trees)
    bark = default_material(**BARK)
    leaf = default_material(**LEAF)
    ground_mat = default_material(r=0.2, g=0.28, b=0.12, roughness=1.0)
    objects = []
    for k in range(trees):
        segs, leaves = stochastic_tree(iterations=int(its[k]), seed=seed + k)
        segs = refine_segments(segs, rings, taper=0.85)
        ts = TubeSet.from_turtle(segs, leaves, sides, 0.18, leaf_material=1, extra=_bank([bark, leaf, ground_mat]))
        objects.append(ts.host_mesh())
    ground = quad_mesh((0, 0, 0), (extent, 0, 0), (0, 0, -extent), ground_mat, normal=(0, 1, 0))
    ground.material_ids[:] = 2
    ground.materials = np.zeros((0,), MATERIAL_DTYPE)
    objects.append(ground)
    inst = []
    pos = rng.uniform(-0.45 * extent, 0.45 * extent, size=(instances, 2))
    yaw = rng.uniform(0.0, 2.0 * math.pi, instances)
    scl = rng.uniform(0.7, 1.3, instances)
    which = rng.integers(0, trees, instances)
    for k in range(instances):
        inst.append((placement(float(pos[k, 0]), float(pos[k, 1]), float(yaw[k]), float(scl[k])), int(which[k])))
    inst.append((placement(0.0, 0.0, 0.0, 1.0), trees))
    scene = InstancedScene(objects, inst)
    az = rng.uniform(0.0, 2.0 * math.pi, views)
    cams = []
    for k in range(views):
        r = 0.47 * extent
        eye = (r * math.sin(az[k]), 6.0, r * math.cos(az[k]))
        cams.append(look_at_camera(eye, (0.0, 4.0, 0.0), fov_y_deg=40.0, aspect=width / height))
    params = default_params(background_r=0.45, background_g=0.55, background_b=0.75, max_path_depth=max_depth,
                            russian_roulette_min_depth=3, min_samples=min_spp, max_samples_per_pixel=max_spp,
                            relative_error_threshold=rel_err, adaptive_criterion=1)
    el = math.radians(35.0)
    sun = dict(direction=(math.cos(el) * 0.6, math.sin(el), math.cos(el) * 0.8), half_angle=SUN_HALF_ANGLE,
               temperature_k=SUN_TEMPERATURE, luminance=3.0 / (2.0 * math.pi * (1.0 - math.cos(SUN_HALF_ANGLE))))
    return scene, cams, params, sun
