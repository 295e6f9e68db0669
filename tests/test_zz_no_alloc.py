"""The allocation-free dot product (ddg_dot_noalloc) against ddg_dot.

This entry point exists for callers that cannot allocate device memory
(graph capture, fixed device-memory budgets); its scratch is a static device
array inside the library.  The file is named so that pytest collects it
last; it also passes when run alone in a fresh process (the first call on the
device performs the one-time address lookup).
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # relative: same float64 accumulation, different summation order


def _noalloc():
    from ddg_b200 import _lib
    L = _lib.lib()
    fn = L.ddg_dot_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return L, fn


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_dot_noalloc_matches_dot_twice(dtype):
    import torch
    from ddg_b200 import _lib
    L, fn = _noalloc()
    dt = getattr(torch, dtype)
    prec = _lib.DDG_FP64 if dtype == "float64" else _lib.DDG_FP32
    g = torch.Generator(device="cuda").manual_seed(7)
    stream = torch.cuda.current_stream().cuda_stream
    for n in (1_966_080, 1_000_003):              # two calls in a row (and a ragged size)
        x = torch.randn(n, dtype=dt, device="cuda", generator=g)
        y = torch.randn(n, dtype=dt, device="cuda", generator=g)
        ref = torch.empty(1, dtype=torch.float64, device="cuda")
        got = torch.empty(1, dtype=torch.float64, device="cuda")
        assert L.ddg_dot(n, prec, x.data_ptr(), y.data_ptr(), ref.data_ptr(), stream) == 0
        assert fn(n, prec, x.data_ptr(), y.data_ptr(), got.data_ptr(), stream) == 0, L.ddg_last_error()
        torch.cuda.synchronize()
        r, v = float(ref.item()), float(got.item())
        scale = float(torch.sum(torch.abs(x.double() * y.double())).item())
        assert abs(v - r) <= TOL * scale, (n, v, r)


def test_dot_noalloc_rejects_oversize():
    L, fn = _noalloc()
    out = np.zeros(1)
    rc = fn(536870912 + 1, 0, 1, 1, out.ctypes.data, None)
    assert rc != 0 and b"exceeds the maximum" in L.ddg_last_error()
