"""pt_trace_soup_noalloc: closest-hit queries for callers that cannot allocate
device memory (hosts whose own allocator owns the whole device, interactive
callbacks that cannot pay an allocation's implicit synchronisation).  Its
results must equal those of the allocating entry point pt_trace_rays on the
same triangles and rays, on two calls in a row (the second call reuses the
shared scratch array the first one left behind), the largest accepted soup
must fit its fixed scratch, and larger inputs must be refused.

This file is collected last on purpose, so that it also runs after every other
test in the same process.
"""
import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from tests.helpers import random_soup, rays_through_bounds

pytestmark = pytest.mark.gpu

MAX_TRIANGLES = 16384  # PT_NOALLOC_MAX_TRIANGLES in include/pt_b200.h


def _lib():
    from lsystemeditor_b200.pathtracer import load_library
    L = load_library()
    vp = C.c_void_p
    L.pt_trace_soup_noalloc.argtypes = [C.c_uint32, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                        C.c_char_p, C.c_size_t]
    L.pt_trace_soup_noalloc.restype = C.c_int
    return L


class _DeviceQuery:
    """Device copies of one soup and one ray batch plus result buffers."""

    def __init__(self, mesh, o, d, tmin, tmax, with_normals=True):
        import torch
        dev = torch.device("cuda", 0)
        m = mesh.contiguous()
        self.triangles = m.triangle_count
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).reshape(-1)).to(dev)
        self.pos, self.nrm, self.uvs = up(m.positions), up(m.normals) if with_normals else None, up(m.uvs)
        self.n = len(o)
        self.o, self.d, self.tmin, self.tmax = up(o), up(d), up(tmin), up(tmax)
        self.hit = torch.zeros(self.n, dtype=torch.uint8, device=dev)
        self.t = torch.zeros(self.n, dtype=torch.float32, device=dev)
        self.tri = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.normal = torch.zeros(3 * self.n, dtype=torch.float32, device=dev)
        self.uv = torch.zeros(2 * self.n, dtype=torch.float32, device=dev)
        self.stream = torch.cuda.current_stream(dev)
        torch.cuda.synchronize(dev)

    def run(self, L):
        import torch
        err = C.create_string_buffer(256)
        nrm = self.nrm.data_ptr() if self.nrm is not None else None
        rc = L.pt_trace_soup_noalloc(self.triangles, self.pos.data_ptr(), nrm, self.uvs.data_ptr(),
                                     self.n, self.o.data_ptr(), self.d.data_ptr(), self.tmin.data_ptr(),
                                     self.tmax.data_ptr(), self.hit.data_ptr(), self.t.data_ptr(), self.tri.data_ptr(),
                                     self.normal.data_ptr(), self.uv.data_ptr(), C.c_void_p(self.stream.cuda_stream),
                                     err, 256)
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize(0)

    def results(self):
        return dict(hit=self.hit.cpu().numpy().astype(bool), t=self.t.cpu().numpy(),
                    tri=self.tri.cpu().numpy().astype(np.uint32), normal=self.normal.cpu().numpy().reshape(-1, 3),
                    uv=self.uv.cpu().numpy().reshape(-1, 2))


def _compare(a, b, label):
    """Bit-exact on hit flags and on every attribute of hits with the same
    triangle id; different ids only as exact-t ties, and rarely."""
    assert np.array_equal(a["hit"], b["hit"]), label
    same = a["hit"] & (a["tri"] == b["tri"])
    diff = np.nonzero(a["hit"] & (a["tri"] != b["tri"]))[0]
    assert np.all(a["t"][diff] == b["t"][diff]), f"{label}: id mismatch without a t tie"
    assert len(diff) <= max(1, len(a["hit"]) // 10000), label
    for k in ("t", "normal", "uv"):
        assert np.array_equal(a[k][same], b[k][same]), (label, k)


def _case(n_tris, seed, n_rays=50_000):
    mesh = random_soup(n_tris, seed=seed, extent=4.0 * (n_tris / 3000.0) ** (1.0 / 3.0))
    o, d = rays_through_bounds(mesh, n_rays, seed=seed + 100)
    rng = np.random.default_rng(seed + 200)
    tmin = np.where(rng.uniform(size=n_rays) < 0.5, 0.0, 0.1).astype(np.float32)
    tmax = np.where(rng.uniform(size=n_rays) < 0.5, 1e6, 5.0).astype(np.float32)
    return mesh, o, d, tmin, tmax


def test_noalloc_trace_matches_allocating_entry_point_twice():
    import torch
    from lsystemeditor_b200.pathtracer import PathTracer
    L = _lib()
    # two calls in a row: a small soup, then the largest accepted one
    cases = [_case(3000, 41), _case(MAX_TRIANGLES, 42)]
    queries = [_DeviceQuery(*c) for c in cases]
    with PathTracer(0) as pt:
        expected = []
        for mesh, o, d, tmin, tmax in cases:
            pt.configure(8, 8, mesh)
            expected.append(pt.trace_rays(o, d, tmin, tmax))
    for k, (q, expect) in enumerate(zip(queries, expected)):
        free0, _ = torch.cuda.mem_get_info(0)
        q.run(L)
        free1, _ = torch.cuda.mem_get_info(0)
        if k > 0:  # the first call on the device may load the module; later calls allocate nothing
            assert free1 >= free0, "device memory was allocated during the call"
        assert expect["hit"].sum() > 1000
        _compare(q.results(), expect, f"call {k + 1}")
    # and once more on the first soup, after the larger one left its data in the scratch array
    queries[0].hit.zero_()
    queries[0].run(L)
    _compare(queries[0].results(), expected[0], "call 3")


def test_noalloc_rejects_oversized_input():
    L = _lib()
    err = C.create_string_buffer(256)
    rc = L.pt_trace_soup_noalloc(MAX_TRIANGLES + 1, None, None, None, 0, None, None, None, None, None, None, None,
                                 None, None, None, err, 256)
    assert rc == 1  # PT_ERR_INVALID_ARGUMENT
    assert b"exceed the maximum of 16384" in err.value


def _face_normal_mesh(mesh):
    """The soup with every vertex normal replaced by the float32 geometric normal (v1 - v0) x (v2 - v0)."""
    m = mesh.contiguous()
    p = m.positions.astype(np.float32)
    e1, e2 = p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]
    g = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1], e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                  e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1).astype(np.float32)
    return type(m)(m.positions, np.repeat(g[:, None, :], 3, axis=1), m.uvs, m.material_ids, m.materials, m.textures)


def test_noalloc_without_normals_reports_face_normals():
    """normals = NULL: the reported normal is the triangle's geometric normal facing the ray, the same
    as the allocating entry point gives for a soup whose vertex normals are the face normals."""
    from lsystemeditor_b200.pathtracer import PathTracer
    L = _lib()
    mesh, o, d, tmin, tmax = _case(4000, 43)
    q = _DeviceQuery(mesh, o, d, tmin, tmax, with_normals=False)
    with PathTracer(0) as pt:
        pt.configure(8, 8, _face_normal_mesh(mesh))
        expect = pt.trace_rays(o, d, tmin, tmax)
    q.run(L)
    got = q.results()
    assert expect["hit"].sum() > 1000
    _compare(got, expect, "no normals")
    assert np.allclose(np.linalg.norm(got["normal"][got["hit"]], axis=1), 1.0, atol=1e-5)


def test_noalloc_scratch_follows_the_context():
    """A module global has its own address in every CUDA context: the scratch address is looked up per
    context (keyed by the context's id), so the query gives the same results in the primary context, in a
    second context of the same device, and in the primary context again.  Runs in a child process that
    drives the contexts through the driver API."""
    from lsystemeditor_b200._build import LIB
    from lsystemeditor_b200.pathtracer import PathTracer
    mesh, o, d, tmin, tmax = _case(2000, 44, n_rays=20_000)
    with PathTracer(0) as pt:
        pt.configure(8, 8, _face_normal_mesh(mesh))
        expect = pt.trace_rays(o, d, tmin, tmax)
    with tempfile.TemporaryDirectory() as tmp:
        inp, out = os.path.join(tmp, "in.npz"), os.path.join(tmp, "out.npz")
        m = mesh.contiguous()
        np.savez(inp, pos=m.positions, uvs=m.uvs, o=o, d=d, tmin=tmin, tmax=tmax, lib=LIB)
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        r = subprocess.run([sys.executable, "-m", "tests.noalloc_contexts", inp, out], cwd=root,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        res = dict(np.load(out))
    for tag in ("primary", "second", "again"):
        got = dict(hit=res[f"{tag}_hit"].astype(bool), t=res[f"{tag}_t"], tri=res[f"{tag}_tri"],
                   normal=res[f"{tag}_normal"].reshape(-1, 3), uv=res[f"{tag}_uv"].reshape(-1, 2))
        _compare(got, expect, tag)
