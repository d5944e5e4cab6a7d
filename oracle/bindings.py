"""ctypes bindings for the two CPU checkers (test infrastructure).

* ``Checker("oracle")`` loads oracle/libpt_oracle.so -- this project's C++
  restatement of the reference render path (FP32 ``orc_*`` and FP64 ``orc64_*``).
* ``Checker("ref")`` loads oracle/_ref/libptref.so -- the reference's own
  hot-path code compiled for the host (only where it could be built).
* ``ReferenceGenerator`` loads oracle/_ref/libptref_gen.so -- the reference's
  L-system, turtle and spline code with its loft restated (scene generator).
* ``ReferenceGpu`` loads oracle/_ref/libptref_gpu.so -- the reference's own
  CUDA render kernels (PathTracer.cu) compiled for sm_100a, driven by the wave
  loop of its render loop; a GPU checker and the GPU bar of the benchmark.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Both libraries expose the same entry points, so a test can run
one case through either and compare.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libpt_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libptref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libptref_gpu.so")
# Where the reference checkout lies; only the build recipes read it (the built
# libraries under oracle/_ref are used where the tree is absent).
REF_ROOT = os.environ.get("LSYSTEM_REFERENCE_ROOT", "/root/reference")

_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)


def _ptr(a: Optional[np.ndarray], t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _vp(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert isinstance(a, np.ndarray), "pass records through _rec() so that they stay alive during the call"
    return C.c_void_p(a.ctypes.data)


def _rec(a):
    """Contiguous array form of a record (np.void rows included); keep the result alive across the call."""
    if a is None:
        return None
    return np.ascontiguousarray(np.array(a) if isinstance(a, np.void) else a)


def build_oracle(force: bool = False) -> str:
    """Compiles the restatement with make (gcc; no reference tree needed)."""
    src = [os.path.join(HERE, f) for f in ("pt_oracle.cpp", "pt_oracle.h")]
    if force or not os.path.exists(ORACLE_SO) or any(os.path.getmtime(s) > os.path.getmtime(ORACLE_SO) for s in src):
        subprocess.run(["make", "-C", HERE, "liboracle"], check=True, stdout=subprocess.DEVNULL)
    return ORACLE_SO


def build_ref() -> Optional[str]:
    """Compiles the reference's own sources for the host where the reference tree exists."""
    if os.path.exists(REF_SO) and not os.path.isdir(REF_ROOT):
        return REF_SO
    if not os.path.isdir(REF_ROOT):
        return None
    src = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "ref_shim", "curand_kernel.h")]
    if not os.path.exists(REF_SO) or any(os.path.getmtime(s) > os.path.getmtime(REF_SO) for s in src):
        subprocess.run(["make", "-C", HERE, "ref", f"REF_ROOT={REF_ROOT}"], check=True, stdout=subprocess.DEVNULL)
    return REF_SO


def build_ref_gpu() -> Optional[str]:
    """Compiles the reference's CUDA render kernels for sm_100a where the reference tree exists."""
    if not os.path.isdir(REF_ROOT):
        return REF_GPU_SO if os.path.exists(REF_GPU_SO) else None
    src = [os.path.join(HERE, "ref_gpu_harness.cu"), os.path.join(HERE, "Makefile")]
    if not os.path.exists(REF_GPU_SO) or any(os.path.getmtime(s) > os.path.getmtime(REF_GPU_SO) for s in src):
        subprocess.run(["make", "-C", HERE, "refgpu", f"REF_ROOT={REF_ROOT}"], check=True, stdout=subprocess.DEVNULL)
    return REF_GPU_SO


REF_GEN_SO = os.path.join(HERE, "_ref", "libptref_gen.so")
WRAPPER_BIN = os.path.join(HERE, "_ref", "wrapper_check")


def build_ref_gen() -> Optional[str]:
    """Compiles the reference's scene generator (LSystemLib, Turtle.cpp, Spline.cpp) for the host."""
    if not os.path.isdir(REF_ROOT):
        return REF_GEN_SO if os.path.exists(REF_GEN_SO) else None
    src = [os.path.join(HERE, "ref_gen_harness.cpp"), os.path.join(HERE, "Makefile")]
    if not os.path.exists(REF_GEN_SO) or any(os.path.getmtime(s) > os.path.getmtime(REF_GEN_SO) for s in src):
        subprocess.run(["make", "-C", HERE, "refgen", f"REF_ROOT={REF_ROOT}"], check=True, stdout=subprocess.DEVNULL)
    return REF_GEN_SO


def build_wrapper() -> Optional[str]:
    """Compiles the C++ PathTracer-shaped wrapper (tests/cpp) against the reference's headers."""
    if not os.path.isdir(REF_ROOT):
        return WRAPPER_BIN if os.path.exists(WRAPPER_BIN) else None
    root = os.path.dirname(HERE)
    src = [os.path.join(root, "tests", "cpp", f) for f in ("wrapper_check.cpp", "PathTracerB200.h")] + \
        [os.path.join(root, "include", "pt_b200.h")]
    if not os.path.exists(WRAPPER_BIN) or any(os.path.getmtime(s) > os.path.getmtime(WRAPPER_BIN) for s in src):
        subprocess.run(["make", "-C", HERE, "wrapper", f"REF_ROOT={REF_ROOT}"], check=True, stdout=subprocess.DEVNULL)
    return WRAPPER_BIN


class Checker:
    def __init__(self, kind: str = "oracle"):
        if kind == "oracle":
            path, self.p = build_oracle(), "orc_"
        elif kind == "ref":
            path = build_ref()
            if path is None or not os.path.exists(path):
                raise FileNotFoundError("reference host build unavailable")
            self.p = "ref_"
        else:
            raise ValueError(kind)
        self.kind = kind
        self.lib = C.CDLL(path)
        L, p = self.lib, self.p
        getattr(L, p + "scene_create").restype = C.c_void_p
        getattr(L, p + "scene_create").argtypes = [C.c_int, _fp, _fp, _fp, _u32p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        getattr(L, p + "scene_destroy").argtypes = [C.c_void_p]
        getattr(L, p + "scene_bvh_node_count").argtypes = [C.c_void_p]
        getattr(L, p + "scene_emissive").argtypes = [C.c_void_p, _u32p, _fp]
        getattr(L, p + "trace_rays").argtypes = [C.c_void_p, C.c_int, _fp, _fp, _fp, _fp, _u8p, _fp, _u32p, _fp, _fp]
        getattr(L, p + "env_create").restype = C.c_void_p
        getattr(L, p + "env_create").argtypes = [C.c_int, C.c_int, _fp]
        getattr(L, p + "env_destroy").argtypes = [C.c_void_p]
        getattr(L, p + "env_tables").argtypes = [C.c_void_p, _fp, _fp]
        getattr(L, p + "render").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                    C.c_uint, _fp, C.c_int, _i32p, C.c_int, _fp, _u32p, _fp, _fp, _u8p, C.c_int]
        getattr(L, p + "trace_pixel").argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                         C.c_int, C.c_int, C.c_uint, _fp, C.c_int, _fp]
        getattr(L, p + "brdf_eval").argtypes = [_fp, _fp, C.c_void_p, C.c_float, C.c_int, _fp, _fp]
        getattr(L, p + "brdf_pdf").restype = C.c_float
        getattr(L, p + "brdf_pdf").argtypes = [_fp, _fp, C.c_void_p, C.c_float, C.c_int, _fp]
        getattr(L, p + "brdf_sample").argtypes = [_fp, _fp, C.c_void_p, C.c_float, C.c_int, C.c_float, C.c_float, _fp, _fp,
                                         _fp, _fp, _i32p]
        getattr(L, p + "brdf_apply_throughput").argtypes = [_fp, _fp, _fp, C.c_void_p, C.c_float, C.c_float, C.c_float, _fp]
        getattr(L, p + "camera_ray").argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_float, _fp, _fp]
        getattr(L, p + "env_sample").argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, _fp, _fp]
        getattr(L, p + "env_pdf").restype = C.c_float
        getattr(L, p + "env_pdf").argtypes = [C.c_void_p, C.c_void_p, _fp]
        getattr(L, p + "env_eval").argtypes = [C.c_void_p, C.c_void_p, _fp, _fp]
        getattr(L, p + "sample_emissive").argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float, _fp, _fp, _fp, _fp]
        getattr(L, p + "is_converged").argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_int, C.c_float]
        getattr(L, p + "brdf_sample_transmit").argtypes = [_fp, _fp, C.c_void_p, C.c_float, C.c_int, C.c_float, C.c_float,
                                                  _fp, _fp, _fp, _i32p]
        getattr(L, p + "lobe_weights").argtypes = [C.c_void_p, _fp]
        getattr(L, p + "resolve_material").argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_int, _fp]
        if kind == "oracle":
            L.orc64_render.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                       C.c_uint, _fp, C.c_int, _i32p, C.c_int, _dp, _u32p, _dp, _dp, _u8p, C.c_int]
            L.orc_trace_rays_bruteforce.argtypes = [C.c_void_p, C.c_int, _fp, _fp, _fp, _fp, _u8p, _fp, _u32p]
            L.orc_reference_seed.restype = C.c_uint
            L.orc_reference_seed.argtypes = [C.c_int, C.c_int, C.c_uint]
            L.orc_render_preview.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, _fp,
                                             C.c_int, _fp]
            L.orc64_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                         _fp, C.c_int, _fp, _dp, C.c_int, C.c_int]
            spec = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint, _fp, C.c_int,
                    C.c_int, _fp, _fp, C.c_int, _fp, C.c_int, _fp, _fp]
            L.orc_render_spectral.argtypes = spec + [_fp, _u32p, _fp, _fp, _u8p, C.c_int]
            L.orc64_render_spectral.argtypes = spec + [_dp, _u32p, _dp, _dp, _u8p, C.c_int]
            L.orc_spec_eval.restype = C.c_float
            L.orc_spec_eval.argtypes = [_fp, C.c_float]
            L.orc_scene_set_emitter_mis.argtypes = [C.c_void_p, C.c_int]
            L.orc_scene_set_adaptive_criterion.argtypes = [C.c_void_p, C.c_int]
            L.orc_scene_set_sun.argtypes = [C.c_void_p, C.c_int, _fp, C.c_float, _fp, C.c_float, C.c_float, _fp, _fp]
            L.orc_hero_lambda.restype = C.c_float
            L.orc_hero_lambda.argtypes = [C.c_uint, C.c_int, C.c_int]

    def fn(self, name):
        # attribute access caches the function object, so argtypes/restype set in __init__ stick
        return getattr(self.lib, self.p + name)

    def max_threads(self) -> int:
        return int(self.fn("max_threads")())

    # -- the reference's spectral helpers (reference build only) -------------
    def ref_spectral_cie(self, lambdas) -> np.ndarray:
        """x-bar, y-bar, z-bar, D65 of Spectral/SpectralCore.h at each wavelength (n x 4)."""
        lam = np.ascontiguousarray(lambdas, np.float32)
        out = np.empty((len(lam), 4), np.float32)
        self.lib.ref_spectral_cie.argtypes = [_fp, C.c_int, _fp]
        self.lib.ref_spectral_cie(_ptr(lam, _fp), len(lam), _ptr(out, _fp))
        return out

    def ref_spectral_xyz_to_srgb(self, xyz) -> np.ndarray:
        a = np.ascontiguousarray(np.asarray(xyz, np.float32).reshape(-1, 3))
        out = np.empty_like(a)
        self.lib.ref_spectral_xyz_to_srgb.argtypes = [_fp, C.c_int, _fp]
        self.lib.ref_spectral_xyz_to_srgb(_ptr(a, _fp), len(a), _ptr(out, _fp))
        return out

    def ref_spectral_sigmoid(self, coef, lambdas) -> np.ndarray:
        c = np.ascontiguousarray(np.asarray(coef, np.float32).reshape(-1, 3))
        lam = np.ascontiguousarray(lambdas, np.float32)
        out = np.empty(len(lam), np.float32)
        self.lib.ref_spectral_sigmoid.argtypes = [_fp, _fp, C.c_int, _fp]
        self.lib.ref_spectral_sigmoid(_ptr(c, _fp), _ptr(lam, _fp), len(lam), _ptr(out, _fp))
        return out

    def spec_eval(self, coef, lam: float) -> float:
        """Spectrum of a coefficient record (c0, c1, c2, scale) at lam nm, FP32 (oracle only)."""
        c = np.ascontiguousarray(coef, np.float32)
        return float(self.lib.orc_spec_eval(_ptr(c, _fp), C.c_float(lam)))

    def hero_lambda(self, seed: int, k: int, nw: int) -> float:
        """Wavelength k of nw of the path with this seed (oracle only)."""
        return float(self.lib.orc_hero_lambda(C.c_uint(seed), int(k), int(nw)))

    # -- scene ------------------------------------------------------------
    def scene(self, mesh) -> "CheckerScene":
        return CheckerScene(self, mesh)

    def env(self, rgb: np.ndarray) -> "CheckerEnv":
        return CheckerEnv(self, rgb)

    # -- BSDF / lights / camera ------------------------------------------
    def brdf_eval(self, normal, wo, material, eta, wi, debug=0):
        material_ = _rec(material)
        out = np.zeros(3, np.float32)
        self.fn("brdf_eval")(_ptr(np.ascontiguousarray(normal, np.float32), _fp),
                             _ptr(np.ascontiguousarray(wo, np.float32), _fp), _vp(material_), C.c_float(eta),
                             int(debug), _ptr(np.ascontiguousarray(wi, np.float32), _fp), _ptr(out, _fp))
        return out

    def brdf_pdf(self, normal, wo, material, eta, wi, debug=0) -> float:
        material_ = _rec(material)
        return float(self.fn("brdf_pdf")(_ptr(np.ascontiguousarray(normal, np.float32), _fp),
                                         _ptr(np.ascontiguousarray(wo, np.float32), _fp), _vp(material_),
                                         C.c_float(eta), int(debug),
                                         _ptr(np.ascontiguousarray(wi, np.float32), _fp)))

    def brdf_sample(self, normal, wo, material, eta, u1, u2, debug=0):
        material_ = _rec(material)
        d = np.zeros(3, np.float32); pdf = np.zeros(1, np.float32); ne = np.zeros(1, np.float32)
        off = np.zeros(3, np.float32); flags = np.zeros(1, np.int32)
        steps = self.fn("brdf_sample")(_ptr(np.ascontiguousarray(normal, np.float32), _fp),
                                       _ptr(np.ascontiguousarray(wo, np.float32), _fp), _vp(material_),
                                       C.c_float(eta), int(debug), C.c_float(u1), C.c_float(u2), _ptr(d, _fp),
                                       _ptr(pdf, _fp), _ptr(ne, _fp), _ptr(off, _fp), _ptr(flags, _i32p))
        f = int(flags[0])
        return dict(direction=d, pdf=float(pdf[0]), valid=bool(f & 1), transmitted=bool(f & 2),
                    subsurface=bool(f & 4), next_eta=float(ne[0]), exit_offset=off, steps=int(steps))

    def brdf_sample_transmit(self, normal, wo, material, eta, u1, u2, debug=0):
        material_ = _rec(material)
        d = np.zeros(3, np.float32); pdf = np.zeros(1, np.float32); ne = np.zeros(1, np.float32)
        flags = np.zeros(1, np.int32)
        self.fn("brdf_sample_transmit")(_ptr(np.ascontiguousarray(normal, np.float32), _fp),
                                        _ptr(np.ascontiguousarray(wo, np.float32), _fp), _vp(material_),
                                        C.c_float(eta), int(debug), C.c_float(u1), C.c_float(u2), _ptr(d, _fp),
                                        _ptr(pdf, _fp), _ptr(ne, _fp), _ptr(flags, _i32p))
        f = int(flags[0])
        return dict(direction=d, pdf=float(pdf[0]), valid=bool(f & 1), transmitted=bool(f & 2),
                    subsurface=bool(f & 4), next_eta=float(ne[0]))

    def lobe_weights(self, material):
        material_ = _rec(material)
        out = np.zeros(4, np.float32)
        self.fn("lobe_weights")(_vp(material_), _ptr(out, _fp))
        return out

    def resolve_material(self, material, u, v, textures=None):
        material_ = _rec(material)
        out = np.zeros(15, np.float32)
        tex = None if textures is None or len(textures) == 0 else np.ascontiguousarray(textures)
        self.fn("resolve_material")(_vp(material_), C.c_float(u), C.c_float(v), _vp(tex),
                                    0 if tex is None else len(tex), _ptr(out, _fp))
        return out

    def brdf_apply_throughput(self, throughput, normal, wo, material, eta, u1, u2):
        material_ = _rec(material)
        out = np.zeros(3, np.float32)
        self.fn("brdf_apply_throughput")(_ptr(np.ascontiguousarray(throughput, np.float32), _fp),
                                         _ptr(np.ascontiguousarray(normal, np.float32), _fp),
                                         _ptr(np.ascontiguousarray(wo, np.float32), _fp), _vp(material_),
                                         C.c_float(eta), C.c_float(u1), C.c_float(u2), _ptr(out, _fp))
        return out

    def camera_ray(self, camera, u, v, l1, l2):
        camera_ = _rec(camera)
        o = np.zeros(3, np.float32); d = np.zeros(3, np.float32)
        self.fn("camera_ray")(_vp(camera_), C.c_float(u), C.c_float(v), C.c_float(l1), C.c_float(l2),
                              _ptr(o, _fp), _ptr(d, _fp))
        return o, d

    # solid background (no environment map): LightSamplingCore.h:56-77, 149-159
    def env_sample_solid(self, params, u1, u2):
        params_ = _rec(params)
        d = np.zeros(3, np.float32); pdf = np.zeros(1, np.float32)
        self.fn("env_sample")(None, _vp(params_), C.c_float(u1), C.c_float(u2), _ptr(d, _fp), _ptr(pdf, _fp))
        return d, float(pdf[0])

    def env_pdf_solid(self, params, d):
        params_ = _rec(params)
        return float(self.fn("env_pdf")(None, _vp(params_), _ptr(np.ascontiguousarray(d, np.float32), _fp)))

    def env_eval_solid(self, params, d):
        params_ = _rec(params)
        out = np.zeros(3, np.float32)
        self.fn("env_eval")(None, _vp(params_), _ptr(np.ascontiguousarray(d, np.float32), _fp), _ptr(out, _fp))
        return out

    def is_converged(self, n, mean, m2, min_samples, thr) -> bool:
        return bool(self.fn("is_converged")(int(n), C.c_float(mean), C.c_float(m2), int(min_samples),
                                            C.c_float(thr)))


class CheckerScene:
    def __init__(self, chk: Checker, mesh):
        self.chk = chk
        m = mesh.contiguous()
        self.mesh = m
        self.h = chk.fn("scene_create")(m.triangle_count, _ptr(m.positions, _fp), _ptr(m.normals, _fp),
                                        _ptr(m.uvs, _fp), _ptr(m.material_ids, _u32p), len(m.materials),
                                        _vp(m.materials) if len(m.materials) else None, len(m.textures),
                                        _vp(m.textures) if len(m.textures) else None)
        if not self.h:
            raise RuntimeError("scene build failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.chk.fn("scene_destroy")(self.h)
            self.h = None

    def bvh_node_count(self) -> int:
        return int(self.chk.fn("scene_bvh_node_count")(self.h))

    def emissive(self):
        n = int(self.chk.fn("scene_emissive")(self.h, None, None))
        idx = np.zeros(max(n, 1), np.uint32)
        cdf = np.zeros(n + 1, np.float32)
        self.chk.fn("scene_emissive")(self.h, _ptr(idx, _u32p), _ptr(cdf, _fp))
        return idx[:n], cdf

    def trace(self, origins, dirs, tmin=None, tmax=None):
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(dirs, np.float32)
        n = o.shape[0]
        tmin = np.zeros(n, np.float32) if tmin is None else np.ascontiguousarray(
            np.broadcast_to(tmin, (n,)), np.float32)
        tmax = np.full(n, 1.0e6, np.float32) if tmax is None else np.ascontiguousarray(
            np.broadcast_to(tmax, (n,)), np.float32)
        hit = np.zeros(n, np.uint8); t = np.zeros(n, np.float32); tri = np.zeros(n, np.uint32)
        nrm = np.zeros((n, 3), np.float32); uv = np.zeros((n, 2), np.float32)
        self.chk.fn("trace_rays")(self.h, n, _ptr(o, _fp), _ptr(d, _fp), _ptr(tmin, _fp), _ptr(tmax, _fp),
                                  _ptr(hit, _u8p), _ptr(t, _fp), _ptr(tri, _u32p), _ptr(nrm, _fp), _ptr(uv, _fp))
        return dict(hit=hit.astype(bool), t=t, tri=tri, normal=nrm, uv=uv)

    def trace_bruteforce(self, origins, dirs, tmin=None, tmax=None):
        assert self.chk.kind == "oracle"
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(dirs, np.float32)
        n = o.shape[0]
        tmin = np.zeros(n, np.float32) if tmin is None else np.ascontiguousarray(
            np.broadcast_to(tmin, (n,)), np.float32)
        tmax = np.full(n, 1.0e6, np.float32) if tmax is None else np.ascontiguousarray(
            np.broadcast_to(tmax, (n,)), np.float32)
        hit = np.zeros(n, np.uint8); t = np.zeros(n, np.float32); tri = np.zeros(n, np.uint32)
        self.chk.lib.orc_trace_rays_bruteforce(self.h, n, _ptr(o, _fp), _ptr(d, _fp), _ptr(tmin, _fp),
                                               _ptr(tmax, _fp), _ptr(hit, _u8p), _ptr(t, _fp), _ptr(tri, _u32p))
        return dict(hit=hit.astype(bool), t=t, tri=tri)

    def sample_emissive(self, u_tri, u1, u2):
        p = np.zeros(3, np.float32); n = np.zeros(3, np.float32); L = np.zeros(3, np.float32)
        pdf = np.zeros(1, np.float32)
        ok = self.chk.fn("sample_emissive")(self.h, C.c_float(u_tri), C.c_float(u1), C.c_float(u2), _ptr(p, _fp),
                                            _ptr(n, _fp), _ptr(L, _fp), _ptr(pdf, _fp))
        return bool(ok), p, n, L, float(pdf[0])

    def render(self, camera, params, width, height, waves, seed_base=1, tape=None, tape_stride=0, env=None,
               pixels=None, state=None, threads=0, fp64=False):
        """Runs adaptive waves like the reference render loop; returns the accumulation state."""
        camera_, params_ = _rec(camera), _rec(params)
        P = width * height
        ft = np.float64 if fp64 else np.float32
        if state is None:
            state = dict(acc=np.zeros((P, 4), ft), counts=np.zeros(P, np.uint32), lum_mean=np.zeros(P, ft),
                         m2=np.zeros(P, ft), converged=np.zeros(P, np.uint8))
        pix = None if pixels is None else np.ascontiguousarray(pixels, np.int32)
        tp = None if tape is None else np.ascontiguousarray(tape, np.float32)
        args = (self.h, env.h if env is not None else None, _vp(camera_), _vp(params_), width, height, waves,
                C.c_uint(seed_base), _ptr(tp, _fp), int(tape_stride), _ptr(pix, _i32p),
                0 if pix is None else len(pix))
        if fp64:
            assert self.chk.kind == "oracle"
            err = self.chk.lib.orc64_render(*args, _ptr(state["acc"], _dp), _ptr(state["counts"], _u32p),
                                            _ptr(state["lum_mean"], _dp), _ptr(state["m2"], _dp),
                                            _ptr(state["converged"], _u8p), int(threads))
        else:
            err = self.chk.fn("render")(*args, _ptr(state["acc"], _fp), _ptr(state["counts"], _u32p),
                                        _ptr(state["lum_mean"], _fp), _ptr(state["m2"], _fp),
                                        _ptr(state["converged"], _u8p), int(threads))
        state["tape_errors"] = int(err)
        return state

    def set_emitter_mis(self, on: bool = True):
        """The emitter MIS estimator (the product's emitter_mis = 1) for this scene's renders."""
        assert self.chk.kind == "oracle"
        self.chk.lib.orc_scene_set_emitter_mis(self.h, 1 if on else 0)
        return self

    def set_adaptive_criterion(self, criterion: int):
        """The product's stop test (adaptive_criterion 0, 1 or 2) for this scene's adaptive renders."""
        assert self.chk.kind == "oracle"
        self.chk.lib.orc_scene_set_adaptive_criterion(self.h, int(criterion))
        return self

    def set_sun(self, direction=None, half_angle=0.0, radiance=(0.0, 0.0, 0.0), temperature_k=0.0, luminance=1.0,
                resp=None, coef=None):
        """Distant light of this scene (orc_scene_set_sun; None removes it).  resp: the 401 x 3 response table
        (blackbody radiance); coef: spectrum coefficients of `radiance` (spectral renders, temperature <= 0)."""
        assert self.chk.kind == "oracle"
        if direction is None:
            self.chk.lib.orc_scene_set_sun(self.h, 0, None, 0.0, None, 0.0, 0.0, None, None)
            return
        d = np.ascontiguousarray(direction, np.float32)
        rad = np.ascontiguousarray(radiance, np.float32)
        rs = None if resp is None else np.ascontiguousarray(resp, np.float32)
        cf = None if coef is None else np.ascontiguousarray(coef, np.float32)
        self.chk.lib.orc_scene_set_sun(self.h, 1, _ptr(d, _fp), C.c_float(half_angle), _ptr(rad, _fp),
                                       C.c_float(temperature_k), C.c_float(luminance), _ptr(rs, _fp), _ptr(cf, _fp))

    def render_spectral(self, camera, params, width, height, waves, spectral, seed_base=1, tape=None, tape_stride=0,
                        env=None, state=None, threads=0, fp64=False):
        """Hero-wavelength render (orc_render_spectral).  `spectral` holds the inputs the product derives from
        the scene: nw, resp (401 x 3), mat (materials x 8), tex (textures x 8), env (texels x 4 or None),
        bg (4)."""
        assert self.chk.kind == "oracle"
        camera_, params_ = _rec(camera), _rec(params)
        P = width * height
        ft = np.float64 if fp64 else np.float32
        if state is None:
            state = dict(acc=np.zeros((P, 4), ft), counts=np.zeros(P, np.uint32), lum_mean=np.zeros(P, ft),
                         m2=np.zeros(P, ft), converged=np.zeros(P, np.uint8))
        tp = None if tape is None else np.ascontiguousarray(tape, np.float32)
        f32 = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)  # noqa: E731
        resp, mat, tex = f32(spectral["resp"]), f32(spectral["mat"]), f32(spectral.get("tex"))
        envc, bg = f32(spectral.get("env")), f32(spectral["bg"])
        keep = (resp, mat, tex, envc, bg)
        args = (self.h, env.h if env is not None else None, _vp(camera_), _vp(params_), width, height, waves,
                C.c_uint(seed_base), _ptr(tp, _fp), int(tape_stride), int(spectral["nw"]), _ptr(resp, _fp),
                _ptr(mat, _fp), 0 if mat is None else len(mat.reshape(-1, 8)), _ptr(tex, _fp),
                0 if tex is None else len(tex.reshape(-1, 8)), _ptr(envc, _fp), _ptr(bg, _fp))
        if fp64:
            err = self.chk.lib.orc64_render_spectral(*args, _ptr(state["acc"], _dp), _ptr(state["counts"], _u32p),
                                                     _ptr(state["lum_mean"], _dp), _ptr(state["m2"], _dp),
                                                     _ptr(state["converged"], _u8p), int(threads))
        else:
            err = self.chk.lib.orc_render_spectral(*args, _ptr(state["acc"], _fp), _ptr(state["counts"], _u32p),
                                                   _ptr(state["lum_mean"], _fp), _ptr(state["m2"], _fp),
                                                   _ptr(state["converged"], _u8p), int(threads))
        del keep
        state["tape_errors"] = int(err)
        return state

    def backward(self, camera, params, width, height, spp, tape, tape_stride, d_image, materials, env=None,
                 threads=0):
        """FP64 path-replay gradient (orc64_backward): d loss / d (r, g, b, roughness, metallic, sheen,
        emission) per material for the image of `spp` samples per pixel replayed from `tape`."""
        assert self.chk.kind == "oracle"
        camera_, params_ = _rec(camera), _rec(params)
        tp = np.ascontiguousarray(tape, np.float32)
        d = np.ascontiguousarray(np.asarray(d_image, np.float32)[..., :3]).reshape(-1)
        assert d.size == 3 * width * height
        g = np.zeros((materials, 7), np.float64)
        err = self.chk.lib.orc64_backward(self.h, env.h if env is not None else None, _vp(camera_), _vp(params_),
                                          width, height, int(spp), _ptr(tp, _fp), int(tape_stride), _ptr(d, _fp),
                                          _ptr(g, _dp), int(materials), int(threads))
        return g, int(err)

    def render_preview(self, camera, params, width, height, tape, tape_stride, env=None):
        """One preview pass (pixel centres, one sample, the caller's params) from a tape [pixel][stride]."""
        assert self.chk.kind == "oracle"
        camera_, params_ = _rec(camera), _rec(params)
        tp = np.ascontiguousarray(tape, np.float32)
        out = np.zeros((height, width, 4), np.float32)
        err = self.chk.lib.orc_render_preview(self.h, env.h if env is not None else None, _vp(camera_), _vp(params_),
                                              width, height, _ptr(tp, _fp), int(tape_stride), _ptr(out, _fp))
        return out, int(err)

    def trace_pixel(self, camera, params, width, height, idx, sample_index, global_seed, tape_row, env=None):
        camera_ = _rec(camera)
        params_ = _rec(params)
        out = np.zeros(3, np.float32)
        row = np.ascontiguousarray(tape_row, np.float32)
        used = self.chk.fn("trace_pixel")(self.h, env.h if env is not None else None, _vp(camera_), _vp(params_),
                                          width, height, idx, sample_index, C.c_uint(global_seed),
                                          _ptr(row, _fp), len(row), _ptr(out, _fp))
        return out, int(used)


class CheckerEnv:
    def __init__(self, chk: Checker, rgb: np.ndarray):
        self.chk = chk
        self.rgb = np.ascontiguousarray(rgb, np.float32)
        self.height, self.width = self.rgb.shape[:2]
        self.h = chk.fn("env_create")(self.width, self.height, _ptr(self.rgb, _fp))

    def __del__(self):
        if getattr(self, "h", None):
            self.chk.fn("env_destroy")(self.h)
            self.h = None

    def tables(self):
        marg = np.zeros(self.height + 1, np.float32)
        row = np.zeros(self.height * (self.width + 1), np.float32)
        self.chk.fn("env_tables")(self.h, _ptr(marg, _fp), _ptr(row, _fp))
        return marg, row

    def sample(self, params, u1, u2):
        params_ = _rec(params)
        d = np.zeros(3, np.float32); pdf = np.zeros(1, np.float32)
        self.chk.fn("env_sample")(self.h, _vp(params_), C.c_float(u1), C.c_float(u2), _ptr(d, _fp), _ptr(pdf, _fp))
        return d, float(pdf[0])

    def pdf(self, params, d):
        params_ = _rec(params)
        return float(self.chk.fn("env_pdf")(self.h, _vp(params_), _ptr(np.ascontiguousarray(d, np.float32), _fp)))

    def eval(self, params, d):
        params_ = _rec(params)
        out = np.zeros(3, np.float32)
        self.chk.fn("env_eval")(self.h, _vp(params_), _ptr(np.ascontiguousarray(d, np.float32), _fp), _ptr(out, _fp))
        return out


def reference_available() -> bool:
    try:
        return build_ref() is not None and os.path.exists(REF_SO)
    except Exception:
        return False


def reference_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


class ReferenceGpu:
    """The reference's megakernel (PathTracer.cu, compiled unchanged for sm_100a)
    driven through its launch wrappers by the wave loop of its render loop
    (oracle/ref_gpu_harness.cu).  Needs a CUDA device."""

    def __init__(self):
        path = build_ref_gpu()
        if path is None or not os.path.exists(path):
            raise FileNotFoundError("reference GPU build unavailable")
        L = self.lib = C.CDLL(path)
        L.refgpu_scene_create.restype = C.c_void_p
        L.refgpu_scene_create.argtypes = [C.c_int, _fp, _fp, _fp, _u32p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                          _dp]
        L.refgpu_scene_destroy.argtypes = [C.c_void_p]
        L.refgpu_scene_bvh_node_count.argtypes = [C.c_void_p]
        L.refgpu_env_create.restype = C.c_void_p
        L.refgpu_env_create.argtypes = [C.c_int, C.c_int, _fp, _fp, _fp]
        L.refgpu_env_destroy.argtypes = [C.c_void_p]
        L.refgpu_render.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, _fp,
                                    _u32p, _fp, _fp, _u8p, _dp]

    def scene(self, mesh) -> "ReferenceGpuScene":
        return ReferenceGpuScene(self, mesh)

    def env(self, rgb: np.ndarray, marginal: np.ndarray, row: np.ndarray) -> "ReferenceGpuEnv":
        return ReferenceGpuEnv(self, rgb, marginal, row)


class ReferenceGpuScene:
    def __init__(self, rg: ReferenceGpu, mesh):
        self.rg = rg
        m = mesh.contiguous()
        self.ms = np.zeros(2, np.float64)
        self.h = rg.lib.refgpu_scene_create(m.triangle_count, _ptr(m.positions, _fp), _ptr(m.normals, _fp),
                                            _ptr(m.uvs, _fp), _ptr(m.material_ids, _u32p), len(m.materials),
                                            _vp(m.materials) if len(m.materials) else None, len(m.textures),
                                            _vp(m.textures) if len(m.textures) else None, _ptr(self.ms, _dp))
        if not self.h:
            raise RuntimeError("reference GPU scene build failed")

    @property
    def build_ms(self) -> float:
        """Host median-split BVH + scene build time of the reference (ms)."""
        return float(self.ms[0])

    @property
    def upload_ms(self) -> float:
        return float(self.ms[1])

    def bvh_node_count(self) -> int:
        return int(self.rg.lib.refgpu_scene_bvh_node_count(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.rg.lib.refgpu_scene_destroy(self.h)
            self.h = None

    def render(self, camera, params, width, height, max_waves=0, env=None):
        """One frame from a cleared accumulator; returns the accumulation state
        and the timing of the wave loop."""
        camera_, params_ = _rec(camera), _rec(params)
        P = width * height
        st = dict(acc=np.zeros((P, 4), np.float32), counts=np.zeros(P, np.uint32), lum_mean=np.zeros(P, np.float32),
                  m2=np.zeros(P, np.float32), converged=np.zeros(P, np.uint8))
        out = np.zeros(5, np.float64)
        rc = self.rg.lib.refgpu_render(self.h, env.h if env is not None else None, _vp(camera_), _vp(params_),
                                       width, height, int(max_waves), _ptr(st["acc"], _fp), _ptr(st["counts"], _u32p),
                                       _ptr(st["lum_mean"], _fp), _ptr(st["m2"], _fp), _ptr(st["converged"], _u8p),
                                       _ptr(out, _dp))
        if rc != 0:
            raise RuntimeError(f"reference GPU render failed at step {rc}")
        st.update(device_ms=float(out[0]), waves=int(out[1]), samples=float(out[2]), wall_ms=float(out[3]),
                  compactions=int(out[4]))
        return st


class ReferenceGpuEnv:
    def __init__(self, rg: ReferenceGpu, rgb, marginal, row):
        self.rg = rg
        h, w = rgb.shape[:2]
        self.rgb = np.ascontiguousarray(rgb, np.float32)
        self.marginal = np.ascontiguousarray(marginal, np.float32)
        self.row = np.ascontiguousarray(row, np.float32)
        self.h = rg.lib.refgpu_env_create(w, h, _ptr(self.rgb, _fp), _ptr(self.marginal, _fp), _ptr(self.row, _fp))
        if not self.h:
            raise RuntimeError("reference GPU environment upload failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.rg.lib.refgpu_env_destroy(self.h)
            self.h = None


def reference_generator_available() -> bool:
    return os.path.exists(REF_GEN_SO)


class ReferenceGenerator:
    """The reference's procedural pipeline on the host (oracle/ref_gen_harness.cpp):
    LSystemEvaluator::evaluate -> turtleExecute -> SplinePath::computeLoftFrames
    -> loft -> root transform."""

    def __init__(self):
        path = build_ref_gen()
        if path is None or not os.path.exists(path):
            raise FileNotFoundError("reference generator build unavailable")
        L = self.lib = C.CDLL(path)
        L.refgen_build.restype = C.c_void_p
        L.refgen_build.argtypes = [C.c_char_p, C.c_int, C.c_ulonglong, _fp, _fp, C.c_int, C.c_int, C.c_float,
                                   C.c_float, C.c_float]
        L.refgen_destroy.argtypes = [C.c_void_p]
        L.refgen_error.restype = C.c_char_p
        L.refgen_error.argtypes = [C.c_void_p]
        L.refgen_counts.argtypes = [C.c_void_p, _i32p]
        L.refgen_times.argtypes = [C.c_void_p, _dp]
        L.refgen_triangles.argtypes = [C.c_void_p, _fp, _fp, _fp, _u32p]
        L.refgen_frames.argtypes = [C.c_void_p, _fp, _u32p, _u32p]

    def build(self, definition: str, iterations: int, seed: int = 0xC0FFEE, rotation_deg=(0.0, 0.0, 0.0),
              translation=(0.0, 0.0, 0.0), sides: int = 32, samples_per_span: int = 4, tension: float = 1.0,
              default_step: float = 500.0, default_radius: float = 100.0) -> dict:
        """Mesh (positions (N,3,3), normals, uvs (N,3,2), segment per triangle), loft frames before the root
        transform ((F,13): position, tangent, normal, binormal, radius; frame_start per lofted segment),
        stage times in ms (lsystem, turtle, spline, loft) and counts."""
        rot = np.ascontiguousarray(rotation_deg, np.float32)
        tr = np.ascontiguousarray(translation, np.float32)
        h = self.lib.refgen_build(definition.encode(), int(iterations), int(seed), _ptr(rot, _fp), _ptr(tr, _fp),
                                  int(sides), int(samples_per_span), float(tension), float(default_step),
                                  float(default_radius))
        try:
            err = self.lib.refgen_error(h).decode()
            if err:
                raise ValueError(f"reference L-system: {err}")
            c = np.zeros(5, np.int32)
            self.lib.refgen_counts(h, _ptr(c, _i32p))
            n, segs, nf = int(c[0]), int(c[1]), int(c[2])
            pos = np.zeros((n, 3, 3), np.float32)
            nrm = np.zeros((n, 3, 3), np.float32)
            uv = np.zeros((n, 3, 2), np.float32)
            seg = np.zeros(max(n, 1), np.uint32)
            self.lib.refgen_triangles(h, _ptr(pos, _fp), _ptr(nrm, _fp), _ptr(uv, _fp), _ptr(seg, _u32p))
            frames = np.zeros((max(nf, 1), 13), np.float32)
            start = np.zeros(segs + 1, np.uint32)
            mats = np.zeros(max(segs, 1), np.uint32)
            self.lib.refgen_frames(h, _ptr(frames, _fp), _ptr(start, _u32p), _ptr(mats, _u32p))
            ms = np.zeros(4, np.float64)
            self.lib.refgen_times(h, _ptr(ms, _dp))
        finally:
            self.lib.refgen_destroy(h)
        return dict(positions=pos, normals=nrm, uvs=uv, segment=seg[:n], frames=frames[:nf], frame_start=start,
                    materials=mats[:segs], skipped=int(c[3]), symbols=int(c[4]),
                    ms=dict(lsystem=ms[0], turtle=ms[1], spline=ms[2], loft=ms[3]))
