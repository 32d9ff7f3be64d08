"""Asynchronous host transfers (clg_field_import_async / export_async / wait).

They have no reference counterpart; the tests pin their ordering contract:
an asynchronous import takes effect before the next operation on the field,
a later synchronous import overrides it, an export captures the field's value
at the time of the call, and a pipelined sequence of solves (source k+1 copied
in and solution k copied out while solve k+1 runs) gives the FP64 true
residual of every solve.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355


def pinned(shape):
    import torch

    return torch.empty(shape, dtype=torch.complex128, pin_memory=True).numpy()


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def lat(ctx, clg):
    return clg.Lattice(ctx, (8, 8, 8, 8))


def gauss(clg, lat, seed):
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    f.InitialField(clg.SOURCE_GAUSS, seed, 2)
    out = f.to_numpy()
    f.close()
    return out


@pytest.mark.parametrize("zero_copy", ["0", "1"])
def test_round_trip_and_order(clg, oracle, monkeypatch, zero_copy):
    monkeypatch.setenv("CLG_ZERO_COPY", zero_copy)
    ctx = clg.Context(0)
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 0xC1A60011, 1)
    a = pinned((lat.volume, 4, 3))
    a[:] = gauss(clg, lat, 51)
    b = pinned((lat.volume, 4, 3))
    b[:] = gauss(clg, lat, 52)
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    # import -> export: exact for FP64 storage
    f.from_numpy_async(a)
    out = pinned((lat.volume, 4, 3))
    f.to_numpy_async(out)
    f.wait()
    np.testing.assert_array_equal(out, a)
    # import, then an operator on the field, then export: D a
    f.from_numpy_async(b)
    f.D(U)
    f.to_numpy_async(out)
    f.wait()
    assert rel(out, oracle.wilson_D(lat.dims, U.CopyDataOut(), b, KAPPA)) < 1e-12
    # an asynchronous import followed by a synchronous one: the later wins
    f.from_numpy_async(a)
    f.from_numpy(b)
    np.testing.assert_array_equal(f.to_numpy(), b)
    # two exports of different values through the same slot
    o1, o2 = pinned((lat.volume, 4, 3)), pinned((lat.volume, 4, 3))
    f.from_numpy(a)
    f.to_numpy_async(o1)
    f.from_numpy(b)
    f.to_numpy_async(o2)
    f.wait()
    np.testing.assert_array_equal(o1, a)
    np.testing.assert_array_equal(o2, b)
    f.close()
    U.close()
    lat.close()
    ctx.close()


@pytest.mark.parametrize("prec,tol", [(1, 1e-7), (2, 1e-3)])
def test_low_precision_import(ctx, clg, lat, prec, tol):
    a = pinned((lat.volume, 4, 3))
    a[:] = gauss(clg, lat, 53)
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, precision=prec, nrhs=2)
    f.from_numpy_async(a, rhs=1)
    out = pinned((lat.volume, 4, 3))
    f.to_numpy_async(out, rhs=1)
    f.wait()
    assert rel(out, a) < tol
    f.close()


@pytest.mark.parametrize("zero_copy", ["0", "1"])
def test_pipelined_solves(clg, oracle, monkeypatch, zero_copy):
    """Source k+1 in and solution k out overlap solve k+1 (two field pairs),
    by copy engine and by SM loads/stores (CLG_ZERO_COPY=1, where a field still
    being read by an export must not be overwritten by the next solve)."""
    monkeypatch.setenv("CLG_ZERO_COPY", zero_copy)
    ctx = clg.Context(0)
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60012, 1, 0.25)
    op = oracle.Operator("WILSON_D", lat.dims, U.CopyDataOut(), KAPPA)
    n = 4
    src = [pinned((lat.volume, 4, 3)) for _ in range(n)]
    dst = [pinned((lat.volume, 4, 3)) for _ in range(n)]
    for k in range(n):
        src[k][:] = gauss(clg, lat, 60 + k)
    bf = [clg.CFieldFermionWilsonSquareSU3(lat, KAPPA) for _ in range(2)]
    xf = [clg.CFieldFermionWilsonSquareSU3(lat, KAPPA) for _ in range(2)]
    S = clg.CSLASolverCG(ctx, inner_precision=clg.HALF)
    bf[0].from_numpy_async(src[0])
    for k in range(n):
        if k + 1 < n:
            bf[(k + 1) % 2].from_numpy_async(src[k + 1])
        info = S.Solve(xf[k % 2], bf[k % 2], U, clg.EFO_F_D)[0]
        assert info["status"] == 0
        xf[k % 2].to_numpy_async(dst[k])
    for f in xf + bf:
        f.wait()
    for k in range(n):
        assert op.true_residual(src[k], dst[k]) <= 1e-10
    for f in xf + bf:
        f.close()
    S.close()
    U.close()
    lat.close()
    ctx.close()


@pytest.mark.parametrize("cls,dims,subset", [("CFieldFermionWilsonSquareSU3", (4, 6, 4, 6), "FULL"),
                                             ("CFieldFermionKSSU3", (6, 4, 6, 4), "FULL"),
                                             ("CFieldFermionWilsonSquareSU3", (4, 4, 6, 6), "EVEN"),
                                             ("CFieldFermionKSSU3", (6, 6, 4, 4), "EVEN")])
@pytest.mark.parametrize("zero_copy", ["0", "1"])
def test_pinned_and_pageable_buffers(clg, monkeypatch, cls, dims, subset, zero_copy):
    """Pinned buffers move by copy engine into a device slot (default) or, with
    CLG_ZERO_COPY=1, by SM loads/stores on the copy stream; pageable ones always
    through the slot.  All give the synchronous import/export's values bit for
    bit, on volumes that are not a multiple of the 128-site transfer tile and
    on one-parity fields (the other parity reads zero)."""
    monkeypatch.setenv("CLG_ZERO_COPY", zero_copy)
    ctx = clg.Context(0)  # reads the switch at creation
    lat = clg.Lattice(ctx, dims)
    C = getattr(clg, cls)
    f = C(lat, 0.1, subset=getattr(clg, subset))
    g = C(lat, 0.1, subset=getattr(clg, subset))
    shape = f.to_numpy().shape
    rng = np.random.default_rng(7)
    for pin in (True, False):
        host = pinned(shape) if pin else np.empty(shape, np.complex128)
        host[:] = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        f.from_numpy_async(host)
        g.from_numpy(host)
        want = g.to_numpy()
        out = pinned(shape) if pin else np.empty(shape, np.complex128)
        f.to_numpy_async(out)
        f.wait()
        np.testing.assert_array_equal(out, want)
        np.testing.assert_array_equal(f.to_numpy(), want)
        if subset != "FULL":
            assert np.count_nonzero(want) == want.size // 2
    f.close()
    g.close()
    lat.close()
    ctx.close()
