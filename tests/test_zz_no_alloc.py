"""clg_dot_noalloc: the inner product for callers that may not allocate device
memory (their own memory pool owns the GPU, or a fixed budget, or a hot loop
that cannot take cudaMalloc's device-wide synchronisation).  Checked through
the C ABI against clg_dot on two calls in a row, with the FP64 tolerance of the
other tests.  This file sorts last so a run that stops at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355


def noalloc_dot(clg, a, b):
    out = np.zeros(2 * a.nrhs)
    st = a.ctx.lib.clg_dot_noalloc(a.h, b.h, C.c_void_p(out.ctypes.data))
    return st, out[0::2] + 1j * out[1::2]


def test_noalloc_dot_matches_dot_twice(ctx, clg):
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    n = 3
    a = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    c = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    for r in range(n):
        a.InitialField(clg.SOURCE_GAUSS, 40 + r, 2, rhs=r)
        b.InitialField(clg.SOURCE_GAUSS, 50 + r, 2, rhs=r)
        c.InitialField(clg.SOURCE_Z2, 60 + r, 3, rhs=r)
    for other in (b, c):  # two calls in a row, different inputs
        want = a.Dot(other)
        st, got = noalloc_dot(clg, a, other)
        assert st == clg.SUCCESS
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    # a single-precision even field (the inner-solver shape) as well
    e1 = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.SINGLE)
    e2 = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.SINGLE)
    e1.InitialField(clg.SOURCE_GAUSS, 70, 2)
    e2.InitialField(clg.SOURCE_GAUSS, 71, 2)
    st, got = noalloc_dot(clg, e1, e2)
    assert st == clg.SUCCESS
    np.testing.assert_allclose(got[0], e1.Dot(e2), rtol=1e-12, atol=0)


def test_noalloc_dot_allocates_nothing(ctx, clg):
    """The property the entry point exists for: after the context is made, calls
    leave the device's free memory unchanged (no allocation, lazy module loading
    included).  Also the 64-right-hand-side limit and FP16 fields."""
    import torch

    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    a = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=64)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=64)
    for r in range(64):
        a.InitialField(clg.SOURCE_GAUSS, 100 + r, 2, rhs=r)
        b.InitialField(clg.SOURCE_Z2, 200 + r, 3, rhs=r)
    h1 = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF)
    h2 = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF)
    h1.InitialField(clg.SOURCE_GAUSS, 72, 2)
    h2.InitialField(clg.SOURCE_GAUSS, 73, 2)
    want64 = a.Dot(b)
    want16 = h1.Dot(h2)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        st, got = noalloc_dot(clg, a, b)
        assert st == clg.SUCCESS
        np.testing.assert_allclose(got, want64, rtol=1e-12, atol=0)
        st, got = noalloc_dot(clg, h1, h2)
        assert st == clg.SUCCESS
        np.testing.assert_allclose(got[0], want16, rtol=1e-12, atol=0)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_noalloc_dot_rejects_too_many_rhs(ctx, clg):
    lat = clg.Lattice(ctx, (4, 4, 4, 4))
    a = clg.CFieldFermionKSSU3(lat, 0.02, nrhs=65)
    st, _ = noalloc_dot(clg, a, a)
    assert st == clg.ERR_BAD_ARG
    assert b"at most 64" in ctx.lib.clg_last_error(ctx.h)
