"""falm_mv_dot_static: the context-free inner product that allocates nothing.

It must give falm_mv_dot's value on the same fields (relative 1e-12 in FP64,
1e-9 in mixed precision, where both sum FP32 products in FP64 in a different
order) and an independent FP64 sum of the interior products computed on the
host, on two calls in a row, without changing the device memory in use, and
it must refuse a grid larger than its fixed partial-sum array.  The free
device memory is sampled after the first call: that call performs the set-up,
which may load the library's device code (and with it the fixed array) under
lazy module loading; the calls after it must leave the free memory unchanged.
This file is collected last so that it also runs after every other GPU test."""
import ctypes

import numpy as np
import pytest

from falm_b200 import _lib as L
from falm_b200 import cases
from falm_b200.api import Context

pytestmark = pytest.mark.gpu


def _args(g, prec, a, b, out, stream):
    return (g.sx, g.sy, g.sz, g.gc, L.FP64 if prec == "fp64" else L.MIXED, ctypes.c_void_p(a.data_ptr()),
            ctypes.c_void_p(b.data_ptr()), ctypes.byref(out), stream)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_static_dot_matches_context_dot(lib_built, prec):
    import torch
    case = cases.small_channel(48, 40, 36, intensity=0.0)
    g = case.grid
    ctx = Context(g, prec)
    rng = np.random.default_rng(5)
    a = torch.as_tensor(rng.standard_normal(g.n), dtype=ctx.dtype, device=ctx.device)
    b = torch.as_tensor(rng.standard_normal(g.n), dtype=ctx.dtype, device=ctx.device)
    ref = ctx.dot(a, b)
    gc = g.gc
    ah = a.double().cpu().numpy().reshape(g.sz, g.sy, g.sx)[gc:-gc, gc:-gc, gc:-gc]
    bh = b.double().cpu().numpy().reshape(g.sz, g.sy, g.sx)[gc:-gc, gc:-gc, gc:-gc]
    host_sum = float(np.sum(ah * bh))       # every product exact in FP64 for FP32 inputs
    lib = L.load()
    out = ctypes.c_double()
    args = _args(g, prec, a, b, out, ctx.stream())
    assert lib.falm_mv_dot_static(*args) == L.FALM_OK          # first call on the device: set-up
    first = out.value
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(ctx.device)[0]
    vals = []
    for _ in range(2):
        out.value = float("nan")
        assert lib.falm_mv_dot_static(*args) == L.FALM_OK
        vals.append(out.value)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(ctx.device)[0] == free0
    tol = 1e-12 if prec == "fp64" else 1e-9
    for v in [first] + vals:
        assert v == pytest.approx(ref, rel=tol)
        assert v == pytest.approx(host_sum, rel=tol)
    ctx.close()


def test_static_dot_refuses_oversize_grid(lib_built):
    import torch
    lib = L.load()
    a = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    out = ctypes.c_double(-1.0)
    # 400 x 400 interior rows > 131072: refused before any device work
    rc = lib.falm_mv_dot_static(8, 404, 404, 2, L.FP64, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                                ctypes.byref(out), None)
    assert rc == 10
    assert out.value == -1.0
    # guide-cell counts outside 1..64 are refused before any arithmetic on them
    for gc in (0, 65, 1 << 30):
        rc = lib.falm_mv_dot_static(8, 8, 8, gc, L.FP64, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                                    ctypes.byref(out), None)
        assert rc == L.FALM_ERR_ARG
