"""Procedural scene ingestion: the host side of the reference's meshSceneBuild.

The reference builds a scene from a list of ProceduralInstance records
(ProceduralTypes.h:72-78: an L-system definition, its iteration count, a root
translation and a yaw/pitch/roll rotation in degrees) with meshSceneBuild
(MeshSceneContent.cpp:5-51), which for each instance evaluates the L-system,
runs the turtle, lofts every segment along its Hermite spline and applies the
root transform (ProceduralMeshBuilder::buildHostMesh,
ProceduralMeshBuilder.cpp:266-330), appending all instances into one mesh.

Here the host side stops at the turtle: each instance's word goes through the
turtle in the reference's start pose, the spline's rings and parallel-
transported frames, and the root transform (rotation, then translation, as
applyRootTransform, ProceduralMeshBuilder.cpp:243-253), and the instances'
tubes are concatenated into one TubeSet, which pt_batch_set_tubes lofts on
the device (or TubeSet.host_mesh on the host).  An instance's word is the
product's module list (scene.expand of an axiom and rules); the text syntax
of LSystemLib is not parsed here.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import scene as S

Module = Tuple[str, tuple]


@dataclass
class ProceduralInstance:
    """One instance of meshSceneBuild's input.  `word` is the evaluated L-system
    (a module list); or give `axiom` + `rules` (+ `iterations`, `seed`) and the
    word is expanded with scene.expand."""
    word: Optional[List[Module]] = None
    axiom: Optional[List[Module]] = None
    rules: Optional[Dict[str, Callable]] = None
    iterations: int = 0
    seed: int = 0
    translation: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rotation_deg: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    material: int = 0  # index into the scene's material bank for this instance's tubes

    def evaluated(self) -> List[Module]:
        if self.word is not None:
            return list(self.word)
        if self.axiom is None:
            raise ValueError("a ProceduralInstance needs a word or an axiom")
        return S.expand(list(self.axiom), dict(self.rules or {}), int(self.iterations), seed=int(self.seed))


@dataclass
class ProceduralBuildParams:
    """The loft parameters of meshSceneBuild (MeshSceneBuildParams /
    ProceduralBuildParams): sides of every tube ring and spline samples per
    span; leaves (the leaf symbol's quads) get `leaf_size` and `leaf_material`."""
    circular_segments: int = 64
    samples_per_span: int = 4
    leaf_symbol: Optional[str] = None
    leaf_size: float = 0.1
    leaf_material: int = 0
    materials: Optional[np.ndarray] = None  # the scene's material bank (pt_material records)
    extra: Optional[S.HostMesh] = None      # triangles appended to the tubes (ground, lights)
    refine: Optional[Callable] = field(default=None, repr=False)  # optional ring refinement of the turtle output


def _translate(segments: Sequence[S.Segment], leaves, t) -> Tuple[List[S.Segment], list]:
    t = np.asarray(t, np.float64)
    if not np.any(t):
        return list(segments), list(leaves)
    out = []
    for sg in segments:
        out.append(S.Segment([np.asarray(p, np.float64) + t for p in sg.points], sg.tangents, list(sg.radii),
                             sg.material, sg.tag, sg.normals, sg.binormals))
    lv = [(np.asarray(p, np.float64) + t, d, u, size) for (p, d, u, size) in leaves]
    return out, lv


def instance_turtle_output(inst: ProceduralInstance, params: ProceduralBuildParams):
    """Framed turtle output of one instance in world space: spline rings and
    frames, root rotation, then root translation."""
    segs, leaves = S.reference_tree(inst.evaluated(), rotation_deg=tuple(inst.rotation_deg),
                                    samples_per_span=params.samples_per_span, leaf_symbol=params.leaf_symbol,
                                    refine=params.refine)
    for sg in segs:
        sg.material = int(inst.material)
    return _translate(segs, leaves, inst.translation)


def build_tubes(instances: Sequence[ProceduralInstance], params: Optional[ProceduralBuildParams] = None) -> S.TubeSet:
    """All instances' tubes in one TubeSet, instance after instance (the order
    in which meshSceneBuild appends their meshes)."""
    params = params or ProceduralBuildParams()
    if not instances:
        raise ValueError("meshSceneBuild needs at least one instance")
    segments, leaves = [], []
    for inst in instances:
        sg, lv = instance_turtle_output(inst, params)
        segments += sg
        leaves += lv
    if not segments:
        raise ValueError("the instances produced no segments")
    extra = params.extra
    if extra is None:
        extra = _empty_mesh(params.materials if params.materials is not None else _default_bank())
    return S.TubeSet.from_turtle(segments, leaves, int(params.circular_segments), float(params.leaf_size),
                                 int(params.leaf_material), extra)


def _default_bank() -> np.ndarray:
    from .records import MATERIAL_DTYPE
    m = np.zeros(1, MATERIAL_DTYPE)
    m["r"] = m["g"] = m["b"] = 0.5
    m["roughness"] = 0.5
    m["ior"] = 1.5
    return m


def _empty_mesh(bank: np.ndarray) -> S.HostMesh:
    """No extra triangles; the material bank of the scene."""
    e = S.HostMesh.empty()
    e.materials = np.asarray(bank)
    return e


# ---------------------------------------------------------------------------
# Stochastic rule choice as the reference's evaluator makes it
# (LSystemEvaluator.cpp:308-347, 386-425, 433-448): one 64-bit Mersenne
# Twister seeded with the evaluation seed; for every symbol, in string order,
# that some rule matches, one uniform draw in [0, total weight) picks the rule
# whose running weight first reaches it.  A symbol without a matching rule is
# copied and draws nothing.
# ---------------------------------------------------------------------------
class ReferenceRng:
    """MT19937-64 (Matsumoto & Nishimura, the std::mt19937_64 parameters) with
    the uniform real draw of std::uniform_real_distribution<double> over it:
    one 64-bit output rounded to double and scaled by 2^-64, then a + u (b - a)."""

    _N, _M = 312, 156
    _MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        mt = [0] * self._N
        mt[0] = seed & self._MASK
        for i in range(1, self._N):
            prev = mt[i - 1]
            mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & self._MASK
        self._mt = mt
        self._i = self._N

    def _twist(self):
        mt, n, m = self._mt, self._N, self._M
        upper, lower = 0xFFFFFFFF80000000, 0x7FFFFFFF
        for i in range(n):
            y = (mt[i] & upper) | (mt[(i + 1) % n] & lower)
            v = mt[(i + m) % n] ^ (y >> 1)
            if y & 1:
                v ^= 0xB5026F5AA96619E9
            mt[i] = v
        self._i = 0

    def next_u64(self) -> int:
        if self._i >= self._N:
            self._twist()
        x = self._mt[self._i]
        self._i += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        return x & self._MASK

    def uniform(self, a: float, b: float) -> float:
        u = float(self.next_u64()) / 18446744073709551616.0
        if u >= 1.0:
            u = np.nextafter(1.0, 0.0)
        return u * (b - a) + a


StochasticRules = Dict[str, List[Tuple[float, Callable[[tuple], List[Module]]]]]


def expand_stochastic(axiom: List[Module], rules: StochasticRules, iterations: int, seed: int) -> List[Module]:
    """Rewrites `axiom` `iterations` times; rules[name] lists the (probability,
    successor(args)) pairs of the rules whose predecessor is `name`, in the
    order the grammar lists them."""
    rng = ReferenceRng(seed)
    word = list(axiom)
    for _ in range(int(iterations)):
        out: List[Module] = []
        for name, args in word:
            cands = rules.get(name)
            if not cands:
                out.append((name, args))
                continue
            weights = [p if (np.isfinite(p) and p > 0.0) else 0.0 for p, _ in cands]
            total = 0.0
            for w in weights:
                total += w
            pick = 0
            if total > 0.0:
                selected = rng.uniform(0.0, total)
                running = 0.0
                pick = len(cands) - 1
                for k, w in enumerate(weights):
                    running += w
                    if selected <= running:
                        pick = k
                        break
            out.extend(cands[pick][1](args))
        word = out
    return word
