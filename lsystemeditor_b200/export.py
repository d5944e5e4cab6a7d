"""File output of scenes and images (headless replacements of the GUI paths).

* ``write_obj``: Wavefront OBJ + MTL of a mesh, in the layout of the
  reference's exporter (PathTracerLib/src/MeshAccel/MeshAccelWavefrontExport.cpp:
  64-142): one ``mat_<i>`` MTL entry per material (Ka = 0.2 Kd, Ks = Kd x
  metallic, Ns = 10 + (1 - roughness) x 990, Ni = ior, d = 1 - transmission,
  Ke = Kd x emission when emissive), ``o scene``, ``usemtl`` on every change of
  material, three vertices + three normals per triangle and ``f a//a b//b c//c``.
  Normals are written as ``vn`` records (the reference passes the multi-character
  constant 'vn' as a char and so writes them with an ``n`` prefix).
* ``write_png``: 8-bit RGBA image (e.g. ``PathTracer.tonemap``) as a PNG file.
"""
from __future__ import annotations

import os
import struct
import zlib

import numpy as np

from .scene import HostMesh


def _f(v: float) -> str:
    return f"{float(v):.6f}"


def write_obj(path: str, mesh: HostMesh, materials=None) -> None:
    """Writes `path` (OBJ) and the MTL file beside it (same base name)."""
    mats = mesh.materials if materials is None else materials
    base = os.path.splitext(os.path.basename(path))[0]
    mtl_path = os.path.join(os.path.dirname(os.path.abspath(path)), base + ".mtl")
    with open(mtl_path, "w") as f:
        f.write("# PathTracer Wavefront MTL export\n\n")
        f32 = np.float32
        for i, m in enumerate(np.atleast_1d(mats)):
            # single-precision arithmetic, as the reference exporter
            r, g, b = f32(m["r"]), f32(m["g"]), f32(m["b"])
            rough = min(max(f32(m["roughness"]), f32(0.0)), f32(1.0))
            met = f32(m["metallic"])
            em = f32(m["emission"]) if f32(m["emission"]) > 0 else f32(0.0)
            opacity = f32(1.0) - min(max(f32(m["transmission"]), f32(0.0)), f32(1.0))
            f.write(f"newmtl mat_{i}\n")
            f.write(f"Ka {_f(r * f32(0.2))} {_f(g * f32(0.2))} {_f(b * f32(0.2))}\n")
            f.write(f"Kd {_f(r)} {_f(g)} {_f(b)}\n")
            f.write(f"Ks {_f(r * met)} {_f(g * met)} {_f(b * met)}\n")
            f.write(f"Ns {_f(f32(10.0) + (f32(1.0) - rough) * f32(990.0))}\n")
            f.write(f"Ni {_f(m['ior'])}\n")
            f.write(f"d {_f(opacity)}\n")
            if em > 0:
                f.write(f"Ke {_f(r * em)} {_f(g * em)} {_f(b * em)}\n")
            f.write("\n")
    pos = mesh.positions.reshape(-1, 3, 3)
    nrm = mesh.normals.reshape(-1, 3, 3)
    mid = mesh.material_ids.reshape(-1)
    lines = ["# PathTracer Wavefront OBJ export", f"mtllib {base}.mtl", "o scene"]
    current = None
    for i in range(pos.shape[0]):
        if mid[i] != current:
            current = mid[i]
            lines.append(f"usemtl mat_{int(current)}")
        for v in pos[i]:
            lines.append(f"v {_f(v[0])} {_f(v[1])} {_f(v[2])}")
        for n in nrm[i]:
            lines.append(f"vn {_f(n[0])} {_f(n[1])} {_f(n[2])}")
        a = 3 * i + 1
        lines.append(f"f {a}//{a} {a + 1}//{a + 1} {a + 2}//{a + 2}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_obj_triangles(path: str):
    """Positions (N, 3, 3) and material names of a file written by write_obj."""
    verts, tris, mats, cur = [], [], [], None
    with open(path) as f:
        for line in f:
            if line.startswith("v "):
                verts.append([float(x) for x in line.split()[1:4]])
            elif line.startswith("usemtl "):
                cur = line.split()[1]
            elif line.startswith("f "):
                tris.append([int(tok.split("//")[0]) - 1 for tok in line.split()[1:4]])
                mats.append(cur)
    v = np.array(verts, np.float64)
    return v[np.array(tris, np.int64)], mats


def write_png(path: str, rgba8: np.ndarray) -> None:
    """8-bit RGBA (H, W, 4) as a PNG (row 0 at the top)."""
    img = np.ascontiguousarray(rgba8, np.uint8)
    h, w, c = img.shape
    assert c == 4
    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))
