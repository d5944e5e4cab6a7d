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
brackets / ``f`` close the current segment.  Each segment's rings and their
frames come from the reference's Hermite spline and parallel transport
(Spline.cpp:102-255, ``spline_frames``), the tree is rotated by the root
transform (ProceduralMeshBuilder.cpp:211-253, ``rotate_turtle_output``) and
every segment is lofted as an n-gon tube with rings at its frames and flat caps
(Loft.cpp:108-155, ``loft``).  It is a scene generator only; the path tracer
consumes whatever mesh it is given.
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
    # ring frames (unit normal and binormal per ring) from spline_frames; None:
    # the loft derives a frame from each ring's tangent
    normals: Optional[List[np.ndarray]] = None
    binormals: Optional[List[np.ndarray]] = None


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
# Spline frames (Spline.cpp:102-255), restated in single precision with the
# reference's operation order: Hermite spans between the turtle states,
# interior samples only on spans that are not straight, parallel-transported
# frames starting from a normal perpendicular to world up.
# ---------------------------------------------------------------------------
_F = np.float32


def _v3(x) -> np.ndarray:
    return np.asarray(x, np.float32).reshape(3)


def _dot(a, b):
    """x*x' + y*y' + z*z' in single precision, left to right (rows of (..., 3))."""
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]).astype(np.float32) + (a[..., 2] * b[..., 2])


def _len(a):
    return np.sqrt(_dot(a, a).astype(np.float32)).astype(np.float32)


def _nrm(a) -> np.ndarray:
    """vecNormalize3: v * (1 / |v|), (0, 0, -1) for a zero vector."""
    a = np.asarray(a, np.float32)
    l = _len(a)
    inv = (np.float32(1.0) / np.where(l > 0, l, np.float32(1.0))).astype(np.float32)
    out = (a * inv[..., None]).astype(np.float32)
    return np.where((l > 0)[..., None], out, np.array([0.0, 0.0, -1.0], np.float32))


def _cross(a, b) -> np.ndarray:
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1).astype(np.float32)


def _initial_normal(t) -> np.ndarray:
    t = _nrm(t)
    up = np.broadcast_to(np.array([0.0, 1.0, 0.0], np.float32), t.shape)
    up = np.where((np.abs(_dot(t, up)) > np.float32(0.95))[..., None], np.array([1.0, 0.0, 0.0], np.float32), up)
    return _nrm(_cross(up, t))


def _transport(t_prev, t_next, n_prev) -> np.ndarray:
    t0, t1 = _nrm(t_prev), _nrm(t_next)
    axis = _cross(t0, t1)
    al = _len(axis)
    if al <= _F(1e-6):
        return n_prev
    n = (axis * _F(_F(1.0) / al)).astype(np.float32)
    ang = _F(np.arcsin(np.float64(min(max(al, _F(-1.0)), _F(1.0)))))
    c, s_ = _F(np.cos(np.float64(ang))), _F(np.sin(np.float64(ang)))
    omc = _F(_F(1.0) - c)
    x, y, z = (_F(v) for v in n_prev)
    m = lambda a, b: _F(a * b)
    # rotation matrix of Spline.cpp:28-36, entry by entry in the reference's order
    r00 = _F(c + m(m(n[0], n[0]), omc)); r01 = _F(m(m(n[0], n[1]), omc) - m(n[2], s_))
    r02 = _F(m(m(n[0], n[2]), omc) + m(n[1], s_))
    r10 = _F(m(m(n[1], n[0]), omc) + m(n[2], s_)); r11 = _F(c + m(m(n[1], n[1]), omc))
    r12 = _F(m(m(n[1], n[2]), omc) - m(n[0], s_))
    r20 = _F(m(m(n[2], n[0]), omc) - m(n[1], s_)); r21 = _F(m(m(n[2], n[1]), omc) + m(n[0], s_))
    r22 = _F(c + m(m(n[2], n[2]), omc))
    return _nrm(np.array([_F(_F(m(r00, x) + m(r01, y)) + m(r02, z)), _F(_F(m(r10, x) + m(r11, y)) + m(r12, z)),
                          _F(_F(m(r20, x) + m(r21, y)) + m(r22, z))], np.float32))


def _hermite(p0, p1, m0, m1, t):
    t = _F(t)
    t2 = _F(t * t)
    t3 = _F(t2 * t)
    h00 = _F(_F(_F(2.0) * t3) - _F(_F(3.0) * t2)) + _F(1.0)
    h10 = _F(t3 - _F(_F(2.0) * t2)) + t
    h01 = _F(_F(-2.0) * t3) + _F(_F(3.0) * t2)
    h11 = _F(t3 - t2)
    return ((p0 * h00 + m0 * h10).astype(np.float32) + (p1 * h01 + m1 * h11).astype(np.float32)).astype(np.float32)


def _hermite_tangent(p0, p1, m0, m1, t):
    t = _F(t)
    t2 = _F(t * t)
    d00 = _F(_F(6.0) * t2) - _F(_F(6.0) * t)
    d10 = _F(_F(_F(3.0) * t2) - _F(_F(4.0) * t)) + _F(1.0)
    d01 = _F(_F(-6.0) * t2) + _F(_F(6.0) * t)
    d11 = _F(_F(3.0) * t2) - _F(_F(2.0) * t)
    return _nrm(((p0 * d00 + m0 * d10).astype(np.float32) + (p1 * d01 + m1 * d11).astype(np.float32)).astype(np.float32))


def spline_frames(seg: "Segment", samples_per_span: int = 4, tension: float = 1.0) -> Optional["Segment"]:
    """SplinePath::buildFromSegment + computeLoftFrames (Spline.cpp:102-255) of one
    turtle segment: returns the segment with its loft rings (positions, unit
    tangents, radii) and ring frames, or None when its spline has no length
    (the reference then builds a sphere, which is not generated here)."""
    if len(seg.points) < 2:
        return None
    ten = _F(tension if tension > 0 else 1.0)
    spans = []
    for i in range(len(seg.points) - 1):
        p0, p1 = _v3(seg.points[i]), _v3(seg.points[i + 1])
        cl = _len((p1 - p0).astype(np.float32))
        spans.append((p0, p1, (_nrm(_v3(seg.tangents[i])) * _F(cl * ten)).astype(np.float32),
                      (_nrm(_v3(seg.tangents[i + 1])) * _F(cl * ten)).astype(np.float32),
                      _F(seg.radii[i]), _F(seg.radii[i + 1]), cl))
    if sum(float(sp[6]) for sp in spans) <= 1e-6:  # totalArcLength
        return None
    per = max(2, samples_per_span)
    pts: List[Tuple[np.ndarray, np.ndarray, np.float32]] = []

    def append(p, t, r):
        if pts and _len((p - pts[-1][0]).astype(np.float32)) <= _F(1e-6):
            return
        pts.append((p, t, r))

    for k, (p0, p1, m0, m1, r0, r1, cl) in enumerate(spans):
        if k == 0:
            append(p0, _nrm(m0), r0)
        refine = False
        if per > 2 and cl > _F(1e-6):
            cd = ((p1 - p0) * _F(_F(1.0) / cl)).astype(np.float32)
            t0, t1 = _nrm(m0), _nrm(m1)
            if _dot(t0, cd) < _F(0.999) or _dot(t1, cd) < _F(0.999) or _dot(t0, t1) < _F(0.999):
                refine = True
            else:
                mid = _hermite(p0, p1, m0, m1, 0.5)
                lin = ((p0 + p1) * _F(0.5)).astype(np.float32)
                refine = _len((mid - lin).astype(np.float32)) > _F(_F(1e-4) * cl)
        if refine:
            for step in range(1, per - 1):
                t = _F(_F(step) / _F(per - 1))
                append(_hermite(p0, p1, m0, m1, t), _hermite_tangent(p0, p1, m0, m1, t), _F(r0 + _F(r1 - r0) * t))
        append(p1, _nrm(m1), r1)
    normals, binormals = [], []
    n = _initial_normal(pts[0][1])
    for i, (p, t, r) in enumerate(pts):
        if i > 0:
            n = _transport(pts[i - 1][1], t, n)
        tn = _nrm(t)
        b = _nrm(_cross(tn, n))
        n = _nrm(_cross(b, tn))
        normals.append(n)
        binormals.append(b)
    return Segment([q[0].astype(np.float64) for q in pts], [_nrm(q[1]).astype(np.float64) for q in pts],
                   [float(q[2]) for q in pts], seg.material, seg.tag,
                   [v.astype(np.float64) for v in normals], [v.astype(np.float64) for v in binormals])


def spline_frames_all(segments: Sequence["Segment"], samples_per_span: int = 4,
                      tension: float = 1.0) -> List["Segment"]:
    """``spline_frames`` of every segment (segments whose spline has no length
    dropped), vectorised over segments with the same state count whose spans
    are all straight -- every span's end tangents within the reference's 0.999
    of its chord and of each other and its Hermite midpoint within 1e-4 chord
    lengths of the chord's (spanNeedsRefinement false), consecutive states
    more than 1e-6 apart, and every transport step a rotation below 1e-6 --
    which then give one ring per state; other segments take the scalar path.
    The operations are the scalar path's, element by element."""
    F = np.float32
    out: List[Optional[Segment]] = [None] * len(segments)
    slow: List[int] = []
    groups: Dict[int, List[int]] = {}
    for i, sg in enumerate(segments):
        groups.setdefault(len(sg.points), []).append(i)
    ten = F(tension if tension > 0 else 1.0)
    for R, idxs in groups.items():
        if R < 2 or max(2, samples_per_span) <= 2:
            slow += idxs
            continue
        P = np.array([np.asarray(segments[i].points, np.float64).reshape(R, 3) for i in idxs]).astype(np.float32)
        T = np.array([np.asarray(segments[i].tangents, np.float64).reshape(R, 3) for i in idxs]).astype(np.float32)
        rad = np.array([np.asarray(segments[i].radii, np.float64).reshape(R) for i in idxs]).astype(np.float32)
        chord = (P[:, 1:] - P[:, :-1]).astype(np.float32)
        cl = _len(chord)                                              # (N, R-1)
        k = (cl * ten).astype(np.float32)[..., None]
        m0 = (_nrm(T[:, :-1]) * k).astype(np.float32)
        m1 = (_nrm(T[:, 1:]) * k).astype(np.float32)
        inv = (F(1.0) / np.where(cl > 0, cl, F(1.0))).astype(np.float32)
        cd = (chord * inv[..., None]).astype(np.float32)
        t0, t1 = _nrm(m0), _nrm(m1)
        mid = _hermite(P[:, :-1], P[:, 1:], m0, m1, 0.5)
        lin = ((P[:, :-1] + P[:, 1:]) * F(0.5)).astype(np.float32)
        straight = ((cl > F(1e-6)) & (_dot(t0, cd) >= F(0.999)) & (_dot(t1, cd) >= F(0.999)) &
                    (_dot(t0, t1) >= F(0.999)) & (_len((mid - lin).astype(np.float32)) <= (F(1e-4) * cl)))
        ok = straight.all(axis=1)
        # loft points: state 0 with the first span's start tangent, then every span's end
        tan = np.concatenate([_nrm(m0[:, :1]), _nrm(m1)], axis=1)      # (N, R, 3)
        n = _initial_normal(tan[:, 0])
        normals = np.empty_like(tan)
        binormals = np.empty_like(tan)
        for r in range(R):
            if r > 0:
                a0, a1 = _nrm(tan[:, r - 1]), _nrm(tan[:, r])
                ok &= _len(_cross(a0, a1)) <= F(1e-6)  # transport keeps the normal
            tn = _nrm(tan[:, r])
            b = _nrm(_cross(tn, n))
            n = _nrm(_cross(b, tn))
            normals[:, r] = n
            binormals[:, r] = b
        for j, i in enumerate(idxs):
            if not ok[j]:
                slow.append(i)
                continue
            sg = segments[i]
            out[i] = Segment([q for q in P[j].astype(np.float64)], [q for q in _nrm(tan[j]).astype(np.float64)],
                             [float(v) for v in rad[j]], sg.material, sg.tag,
                             [q for q in normals[j].astype(np.float64)], [q for q in binormals[j].astype(np.float64)])
    for i in slow:
        out[i] = spline_frames(segments[i], samples_per_span, tension)
    return [sg for sg in out if sg is not None]


def _rotate_about(v: np.ndarray, axis, deg: float) -> np.ndarray:
    """rotateAroundAxis (ProceduralMeshBuilder.cpp:213-226) in double, rows of v."""
    a = np.asarray(axis, np.float64)
    ang = float(np.float32(deg) * np.float32(0.0174532925))
    c, s_ = math.cos(ang), math.sin(ang)
    d = v @ a
    return v * c + np.cross(a, v) * s_ + np.outer(d, a) * (1.0 - c)


def rotate_yaw_pitch_roll(v: np.ndarray, rotation_deg) -> np.ndarray:
    """rotateYawPitchRoll (ProceduralMeshBuilder.cpp:228-241): yaw about +Y, then
    pitch about +X, then roll about +Z (angles in degrees, skipped when ~0)."""
    v = np.asarray(v, np.float64).reshape(-1, 3)
    for deg, axis in zip(rotation_deg, ((0.0, 1.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0))):
        if abs(deg) > 1e-6:
            v = _rotate_about(v, axis, deg)
    return v


def rotate_turtle_output(segments: Sequence["Segment"], leaves, rotation_deg) -> Tuple[List["Segment"], list]:
    """The root transform of ProceduralMeshBuilder (applyRootTransform,
    ProceduralMeshBuilder.cpp:243-253) applied to ring centres, tangents and
    frames, and to leaf frames, instead of to the lofted vertices (a rotation
    commutes with the loft)."""
    out = []
    for sg in segments:
        rot = lambda xs: [r for r in rotate_yaw_pitch_roll(np.array(xs), rotation_deg)] if xs is not None else None
        out.append(Segment(rot(sg.points), rot(sg.tangents), list(sg.radii), sg.material, sg.tag, rot(sg.normals),
                           rot(sg.binormals)))
    lv = []
    for (p, t, u, size) in leaves:
        q = rotate_yaw_pitch_roll(np.array([p, t, u]), rotation_deg)
        lv.append((q[0], q[1], q[2], size))
    return out, lv


def frame_tree(segments: Sequence["Segment"], leaves, rotation_deg=(0.0, 90.0, 0.0), samples_per_span: int = 4):
    """Spline frames of turtle output in the reference's start pose, then the
    root rotation (the default +90 degree pitch turns heading -Z to +Y)."""
    return rotate_turtle_output(spline_frames_all(segments, samples_per_span), leaves, rotation_deg)


def reference_tree(word: List[Module], rotation_deg=(0.0, 90.0, 0.0), samples_per_span: int = 4,
                   leaf_symbol: Optional[str] = None, refine: Optional[Callable] = None):
    """The reference's procedural pipeline on a symbol string: turtle from its
    default pose (heading -Z, up +Y), optional ring refinement, spline frames,
    root rotation (the default pitch of +90 degrees turns the heading to +Y)."""
    segs, leaves = turtle(word, leaf_symbol=leaf_symbol)
    if refine is not None:
        segs = refine(segs)
    return rotate_turtle_output(spline_frames_all(segs, samples_per_span), leaves, rotation_deg)


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


def angle_table(sides: int) -> Tuple[np.ndarray, np.ndarray]:
    """cos / sin of side k's angle k * 6.283185307f / sides, the angle in single
    precision as Loft.cpp:25 computes it, the cosine and sine rounded to single
    precision; returned in double (the loft's arithmetic)."""
    k = np.arange(sides, dtype=np.float32)
    ang = ((k * np.float32(6.283185307)) / np.float32(sides)).astype(np.float64)
    return (np.cos(ang).astype(np.float32).astype(np.float64), np.sin(ang).astype(np.float32).astype(np.float64))


def loft(segments: Sequence[Segment], sides: int = 8, material_ids: Optional[Sequence[int]] = None) -> HostMesh:
    """buildLoftHostMeshFromFrames (Loft.cpp:108-155) of every segment, in double:
    per ring, vertex k = centre + radius (normal cos_k + binormal sin_k) with the
    segment's frames (or, for a segment without frames, a frame derived from the
    ring tangent); side walls ring by ring (two triangles per side, the seam
    vertex shared with side 0, u = k / sides, v = ring / (rings - 1)), then the
    start and end caps interleaved per side (normals -/+ the unit tangent, rim
    uvs 0.5 + 0.5 (sin, cos), centre 0.5).  Vectorised over segments with the
    same ring count; the device loft (pt_batch_set_tubes) computes the same."""
    groups: Dict[int, List[int]] = {}
    order: List[int] = []
    for i, s in enumerate(segments):
        groups.setdefault(len(s.points), []).append(i)
    cs, sn = angle_table(sides)
    nxt = (np.arange(sides) + 1) % sides
    cap_uv = np.stack([(0.5 + 0.5 * sn).astype(np.float32), (0.5 + 0.5 * cs).astype(np.float32)], -1)  # (sides, 2)
    per_seg_pos, per_seg_nrm, per_seg_uv = {}, {}, {}
    for rings, idxs in groups.items():
        P = np.array([[segments[i].points[k] for k in range(rings)] for i in idxs], np.float64)      # (S, R, 3)
        T = np.array([[segments[i].tangents[k] for k in range(rings)] for i in idxs], np.float64)
        Rr = np.array([[segments[i].radii[k] for k in range(rings)] for i in idxs], np.float64)     # (S, R)
        framed = segments[idxs[0]].normals is not None
        if framed:
            A = np.array([[segments[i].normals[k] for k in range(rings)] for i in idxs], np.float64)
            B = np.array([[segments[i].binormals[k] for k in range(rings)] for i in idxs], np.float64)
            U = T / np.linalg.norm(T, axis=-1, keepdims=True)
        else:
            if rings > 1:
                T[:, -1] = T[:, -2]
            A, B = _perp_frames(T)
            U = T / np.linalg.norm(T, axis=-1, keepdims=True)
        dirs = A[:, :, None, :] * cs[None, None, :, None] + B[:, :, None, :] * sn[None, None, :, None]  # (S,R,C,3)
        ringp = P[:, :, None, :] + dirs * Rr[:, :, None, None]
        S = len(idxs)
        tris_pos, tris_nrm, tris_uv = [], [], []
        span = float(max(rings - 1, 1))
        for r in range(rings - 1):
            v0, v1 = r / span, (r + 1) / span
            for k in range(sides):
                k1 = int(nxt[k])
                u0, u1 = k / sides, (k + 1) / sides
                tris_pos += [np.stack([ringp[:, r, k], ringp[:, r, k1], ringp[:, r + 1, k]], 1),
                             np.stack([ringp[:, r, k1], ringp[:, r + 1, k1], ringp[:, r + 1, k]], 1)]
                tris_nrm += [np.stack([dirs[:, r, k], dirs[:, r, k1], dirs[:, r + 1, k]], 1),
                             np.stack([dirs[:, r, k1], dirs[:, r + 1, k1], dirs[:, r + 1, k]], 1)]
                uvq = np.array([[[u0, v0], [u1, v0], [u0, v1]], [[u1, v0], [u1, v1], [u0, v1]]], np.float64)
                uvq = uvq.astype(np.float32)
                tris_uv += [np.broadcast_to(uvq[0], (S, 3, 2)), np.broadcast_to(uvq[1], (S, 3, 2))]
        c0, c1 = P[:, 0], P[:, rings - 1]
        n0 = np.broadcast_to(-U[:, 0][:, None, :], (S, 3, 3))
        n1 = np.broadcast_to(U[:, rings - 1][:, None, :], (S, 3, 3))
        for k in range(sides):
            k1 = int(nxt[k])
            tris_pos.append(np.stack([c0, ringp[:, 0, k1], ringp[:, 0, k]], 1))
            tris_nrm.append(n0)
            tris_uv.append(np.broadcast_to(np.array([[0.5, 0.5], cap_uv[k1], cap_uv[k]], np.float32), (S, 3, 2)))
            tris_pos.append(np.stack([c1, ringp[:, rings - 1, k], ringp[:, rings - 1, k1]], 1))
            tris_nrm.append(n1)
            tris_uv.append(np.broadcast_to(np.array([[0.5, 0.5], cap_uv[k], cap_uv[k1]], np.float32), (S, 3, 2)))
        pos = np.stack(tris_pos, 1)     # (S, per, 3, 3)
        nrm = np.stack(tris_nrm, 1)
        uv = np.stack(tris_uv, 1)
        for j, i in enumerate(idxs):
            per_seg_pos[i], per_seg_nrm[i], per_seg_uv[i] = pos[j], nrm[j], uv[j]
    if not segments:
        return HostMesh.empty()
    order = list(range(len(segments)))
    mids = np.concatenate([np.full(len(per_seg_pos[i]), segments[i].material if material_ids is None
                                   else material_ids[i], np.uint32) for i in order])
    return HostMesh(np.concatenate([per_seg_pos[i] for i in order]).astype(np.float32),
                    np.concatenate([per_seg_nrm[i] for i in order]).astype(np.float32),
                    np.concatenate([per_seg_uv[i] for i in order]).astype(np.float32), mids,
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
    frames: Optional[np.ndarray] = None  # (R, 6) float64 ring normal + binormal, or None

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
        frames = None
        if segments and all(sg.normals is not None for sg in segments):
            frames = np.concatenate([np.concatenate([np.array(sg.normals, np.float64).reshape(-1, 3),
                                                     np.array(sg.binormals, np.float64).reshape(-1, 3)], 1)
                                     for sg in segments])
        return TubeSet(ring_start, pts, tans, rad, mats, int(sides), lv, float(leaf_size), int(leaf_material),
                       extra, frames)

    @property
    def triangle_count(self) -> int:
        return 2 * self.sides * len(self.radii) + 2 * len(self.leaves) + self.extra.triangle_count

    def cos_sin(self) -> np.ndarray:
        """The loft's angle table (``angle_table``), interleaved cos / sin, with
        entry `sides` repeating entry 0 (the seam)."""
        cs, sn = angle_table(self.sides)
        t = np.stack([cs, sn], -1)
        return np.concatenate([t, t[:1]]).reshape(-1)

    def segments(self) -> List[Segment]:
        out = []
        for t in range(len(self.materials)):
            a, b = int(self.ring_start[t]), int(self.ring_start[t + 1])
            nb = (None, None) if self.frames is None else (list(self.frames[a:b, 0:3]), list(self.frames[a:b, 3:6]))
            out.append(Segment(list(self.points[a:b]), list(self.tangents[a:b]), list(self.radii[a:b]),
                               int(self.materials[t]), 0, nb[0], nb[1]))
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

    The reference pipeline (``reference_tree``): the turtle starts heading -Z
    with up +Y, the spline frames and the loft follow Spline.cpp / Loft.cpp, and
    the root transform's +90 degree pitch turns the tree to head +Y with up +Z,
    so Yaw bends the branches in the XY plane.
    """
    return loft(bracketed_ol_segments(iterations, angle, length, radius), sides)


def bracketed_ol_segments(iterations: int = 4, angle: float = 25.7, length: float = 0.1,
                          radius: float = 0.02) -> List[Segment]:
    """The framed, root-rotated tube segments of ``bracketed_ol_tree``."""
    def rule(args, _rng):
        h, r = args
        F = ("F", (h, r))
        return [F, ("[", ()), ("Yaw", (angle,)), F, ("]", ()), F, ("[", ()), ("Yaw", (-angle,)), F, ("]", ()), F]
    word = expand([("F", (length, radius))], {"F": rule}, iterations)
    segs, _ = reference_tree(word)
    return segs


def stochastic_tree(iterations: int = 7, seed: int = 7, angle: float = 22.5, jitter: float = 5.0,
                    length: float = 0.8, radius: float = 0.08, length_decay: float = 0.9, radius_decay: float = 0.7):
    """3D stochastic L-system tree: axiom A,
        A -> F [&+A] [&-A] [^A]   (p = 0.6)
        A -> F [&A] [^/A]         (p = 0.4)
    with + / - = Yaw(+-a), & / ^ = Pitch(+-a), / = Roll(a), a = angle +- uniform jitter
    (drawn per symbol from a seeded generator and baked into the successor), segment
    length x length_decay and radius x radius_decay per depth.  Terminal A's carry
    a leaf.  Returns (segments, leaves) from the turtle in the reference's start
    pose (heading -Z, up +Y); ``frame_tree`` adds the spline frames and the root
    rotation that turns it to head +Y.
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
    return turtle(word, leaf_symbol="Leaf")


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
    segs, leaves = frame_tree(refine_segments(segs, rings, taper=taper), leaves)
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
    segs, _ = reference_tree(word)
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
    segs = bracketed_ol_segments()
    bark = default_material(r=0.35, g=0.22, b=0.12, roughness=0.8, metallic=0.0)
    tree = loft(segs, 8)
    tree.materials = np.array([bark], MATERIAL_DTYPE)
    ground = quad_mesh((0, 0, 0), (10, 0, 0), (0, 0, -10),
                       default_material(r=0.5, g=0.5, b=0.5, roughness=1.0), normal=(0, 1, 0))
    light = quad_mesh((0, 5, 1.5), (1, 0, 0), (0, 0, 1),
                      default_material(r=1.0, g=1.0, b=1.0, emission=10.0), normal=(0, -1, 0))
    mesh = HostMesh.concat([tree, ground, light])
    tubes = TubeSet.from_turtle(segs, [], 8, 0.0, 0, extra=HostMesh.concat([_bank([bark]), ground, light]))
    lo, hi = tree.bounds()
    center = (lo + hi) * 0.5
    extent = float(np.max(hi - lo))
    dist = extent * 0.5 / math.tan(math.radians(20.0)) * 1.15
    cam = look_at_camera((center[0], center[1], center[2] + dist), center, fov_y_deg=40.0,
                         aspect=width / height)
    params = default_params(background_r=0.0, background_g=0.0, background_b=0.0, max_path_depth=max_depth,
                            russian_roulette_min_depth=3, min_samples=spp, max_samples_per_pixel=spp)
    return SceneSpec("plain-small: 2D bracketed OL-system, 625 segments, 256x256, 64 spp, depth 8",
                     mesh, cam, params, width, height, spp, tubes)


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
        segs, leaves = frame_tree(refine_segments(segs, rings, taper=0.85), leaves)
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
