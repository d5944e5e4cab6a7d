"""Child process of tests/test_zz_no_alloc.py: pt_trace_soup_noalloc in two
CUDA contexts of one device, driven through the CUDA driver API (no torch).

    python -m tests.noalloc_contexts <inputs.npz> <outputs.npz>

The scratch array of the no-alloc entry point is a module global, and a
module global has its own address in every context the module is loaded
into.  The child runs the same query in the device's primary context, then in
a second context it creates (with its own device buffers), then in the
primary context again, and saves the three results; the parent compares each
with the allocating entry point's.
"""
import ctypes as C
import sys

import numpy as np


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with CUresult {rc}")


class _Driver:
    def __init__(self):
        self.cu = C.CDLL("libcuda.so.1")
        _check(self.cu.cuInit(0), "cuInit")
        self.dev = C.c_int(0)
        _check(self.cu.cuDeviceGet(C.byref(self.dev), 0), "cuDeviceGet")

    def alloc(self, nbytes):
        p = C.c_uint64(0)
        _check(self.cu.cuMemAlloc_v2(C.byref(p), C.c_size_t(max(nbytes, 4))), "cuMemAlloc")
        return p.value

    def upload(self, a):
        a = np.ascontiguousarray(a)
        p = self.alloc(a.nbytes)
        _check(self.cu.cuMemcpyHtoD_v2(C.c_uint64(p), a.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes)), "HtoD")
        return p

    def download(self, p, like):
        out = np.empty_like(like)
        _check(self.cu.cuMemcpyDtoH_v2(out.ctypes.data_as(C.c_void_p), C.c_uint64(p), C.c_size_t(out.nbytes)), "DtoH")
        return out

    def free(self, p):
        _check(self.cu.cuMemFree_v2(C.c_uint64(p)), "cuMemFree")


def _query(drv, lib, inp):
    """Uploads the soup and rays into the current context, runs the no-alloc query, returns the results."""
    n = len(inp["tmin"])
    tris = inp["pos"].size // 9
    bufs = {k: drv.upload(inp[k].astype(np.float32).reshape(-1)) for k in ("pos", "uvs", "o", "d", "tmin", "tmax")}
    outs = {"hit": np.zeros(n, np.uint8), "t": np.zeros(n, np.float32), "tri": np.zeros(n, np.uint32),
            "normal": np.zeros(3 * n, np.float32), "uv": np.zeros(2 * n, np.float32)}
    obufs = {k: drv.upload(v) for k, v in outs.items()}
    err = C.create_string_buffer(256)
    vp = C.c_void_p
    rc = lib.pt_trace_soup_noalloc(C.c_uint32(tris), vp(bufs["pos"]), None, vp(bufs["uvs"]), C.c_int(n),
                                   vp(bufs["o"]), vp(bufs["d"]), vp(bufs["tmin"]), vp(bufs["tmax"]),
                                   vp(obufs["hit"]), vp(obufs["t"]), vp(obufs["tri"]), vp(obufs["normal"]),
                                   vp(obufs["uv"]), None, err, C.c_size_t(256))
    if rc != 0:
        raise RuntimeError(f"pt_trace_soup_noalloc: {rc} {err.value.decode()}")
    _check(drv.cu.cuCtxSynchronize(), "cuCtxSynchronize")
    res = {k: drv.download(obufs[k], v) for k, v in outs.items()}
    for p in list(bufs.values()) + list(obufs.values()):
        drv.free(p)
    return res


def main(inp_path, out_path):
    inp = dict(np.load(inp_path))
    drv = _Driver()
    lib = C.CDLL(str(inp["lib"]))
    lib.pt_trace_soup_noalloc.restype = C.c_int
    primary = C.c_void_p()
    _check(drv.cu.cuDevicePrimaryCtxRetain(C.byref(primary), drv.dev), "cuDevicePrimaryCtxRetain")
    _check(drv.cu.cuCtxSetCurrent(primary), "cuCtxSetCurrent")
    first = _query(drv, lib, inp)
    other = C.c_void_p()
    _check(drv.cu.cuCtxCreate_v2(C.byref(other), 0, drv.dev), "cuCtxCreate")  # becomes current
    second = _query(drv, lib, inp)
    _check(drv.cu.cuCtxSetCurrent(primary), "cuCtxSetCurrent")
    _check(drv.cu.cuCtxDestroy_v2(other), "cuCtxDestroy")
    third = _query(drv, lib, inp)
    out = {}
    for tag, r in (("primary", first), ("second", second), ("again", third)):
        for k, v in r.items():
            out[f"{tag}_{k}"] = v
    np.savez(out_path, **out)
    _check(drv.cu.cuDevicePrimaryCtxRelease_v2(drv.dev), "cuDevicePrimaryCtxRelease")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
