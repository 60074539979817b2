"""
cms_nearest_dots_noalloc -- the nearest-dot search for callers that cannot
allocate GPU memory (a framework or application that owns every device
allocation through its own pool, plugins it hosts, real-time loops that must
not meet cudaMalloc's synchronisation): inputs and outputs are the caller's
device buffers and the scratch is a fixed device array inside the library.

Checked through the C ABI against the allocating entry point cms_nearest_dots
on two calls in a row (the shared scratch keeps the previous call's contents,
so the second call must not depend on it), that a warm call leaves the
device's free memory unchanged, plus the size limit.  Collected last so that a run stopping at the first
failure has run everything else.
"""

import ctypes

import numpy as np
import pytest

from parity import exact

pytestmark = pytest.mark.gpu

MAX_POINTS = 3836 * 512


def _lib():
    from cms_cuda import _lib as L
    lib = L.load()
    f = lib.cms_nearest_dots_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int32
    return L, f


def _call(f, q, r, with_index=True):
    """One call through the C ABI; also returns the device's free memory right after it."""
    import torch
    qd = torch.from_numpy(q).cuda()
    rd = torch.from_numpy(r).cuda()
    d2 = torch.empty(len(q), dtype=torch.float64, device="cuda")
    idx = torch.empty(len(q), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = f(qd.data_ptr(), len(q), rd.data_ptr(), len(r), d2.data_ptr(), idx.data_ptr() if with_index else None,
           stream)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return st, d2.cpu().numpy(), idx.cpu().numpy(), (free0, free1)


def test_matches_allocating_entry_point_twice():
    L, f = _lib()
    ctx = L.Context(0)
    rng = np.random.default_rng(7)
    for call, (nq, nr) in enumerate([(2500, 6000), (900, 12000)]):
        q = rng.uniform(-25, 25, (nq, 3))
        r = rng.uniform(-25, 25, (nr, 3))
        r[nr - 1] = r[3]                      # exact tie: the first index wins
        q[0] = r[3]
        st, d2, idx, (free0, free1) = _call(f, q, r)
        assert st == 0, f"call {call}: status {st}"
        if call > 0:
            # the scratch is static: a warm call leaves the device's free memory as it was
            assert free1 == free0, (free0, free1)
        ref_d2, ref_idx = ctx.nearest_dots(q, r)
        exact(f"call {call} min d2", d2, ref_d2)
        exact(f"call {call} argmin", idx, ref_idx)
        assert idx[0] == 3 and d2[0] == 0.0


def test_without_indices_and_size_limit():
    L, f = _lib()
    ctx = L.Context(0)
    rng = np.random.default_rng(8)
    q = rng.uniform(-10, 10, (300, 3))
    r = rng.uniform(-10, 10, (400, 3))
    st, d2, _, _ = _call(f, q, r, with_index=False)
    assert st == 0
    exact("min d2 (no index)", d2, ctx.nearest_dots(q, r)[0])
    # past the fixed scratch: rejected before any launch, outputs untouched
    import torch
    dummy = torch.zeros(3, dtype=torch.float64, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    st = f(dummy.data_ptr(), MAX_POINTS, dummy.data_ptr(), 1, out.data_ptr(), None, None)
    assert st == -1
    assert out.item() == -1.0
