"""The LSD radix sort behind the GPU BVH build (pt_radix_sort_pairs, through
the C ABI) against numpy's stable sort: keys AND values bit for bit, so equal
keys keep their input order; ragged sizes around the 2048-key tile, many
duplicate keys, the 30 bits of the Morton codes and the full 32 bits."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sort(keys, vals, bits):
    import torch
    from lsystemeditor_b200.pathtracer import load_library
    L = load_library()
    dev = torch.device("cuda", 0)
    n = len(keys)
    k = torch.from_numpy(keys.view(np.int32)).to(dev)
    v = torch.from_numpy(vals.view(np.int32)).to(dev)
    ko = torch.empty_like(k)
    vo = torch.empty_like(v)
    tb = int(L.pt_radix_sort_temp_bytes(n))
    temp = torch.empty(max(tb, 1), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = L.pt_radix_sort_pairs(k.data_ptr(), v.data_ptr(), ko.data_ptr(), vo.data_ptr(), n, bits, temp.data_ptr(),
                               tb, C.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize(dev)
    assert np.array_equal(k.cpu().numpy().view(np.uint32), keys), "input keys changed"
    return ko.cpu().numpy().view(np.uint32), vo.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 7, 2047, 2048, 2049, 100_003, 1 << 20])
@pytest.mark.parametrize("bits", [30, 32])
def test_radix_sort_matches_stable_sort(n, bits):
    rng = np.random.default_rng(n + bits)
    hi = (1 << bits) - 1
    keys = rng.integers(0, hi, n, dtype=np.uint64, endpoint=True).astype(np.uint32)
    keys[rng.uniform(size=n) < 0.3] = keys[0]        # a heavy duplicate
    keys[rng.uniform(size=n) < 0.2] &= np.uint32(0xFFFF0000 & hi)  # shared high digits
    vals = np.arange(n, dtype=np.uint32)
    ks, vs = _sort(keys, vals, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(ks, keys[order])
    assert np.array_equal(vs, vals[order])


def test_radix_sort_rejects_bad_arguments():
    from lsystemeditor_b200.pathtracer import load_library
    L = load_library()
    assert L.pt_radix_sort_pairs(None, None, None, None, 10, 30, None, 0, None) == 1
    assert L.pt_radix_sort_pairs(None, None, None, None, 0, 30, None, 0, None) == 0
