"""Parity of the sm_100a operators with the FP64 oracle, through the C ABI.

Tolerances (relative, norm-wise |a - b| / |b|): FP64 1e-12 (the required FP64
Dslash bound), FP32 2e-6, FP16 storage 5e-3.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
KAPPA = 0.1355


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def lat8(ctx, clg):
    return clg.Lattice(ctx, (8, 8, 8, 8))


def make_gauge(clg, lat, kind="haar", seed=0xC1A60000, eps=0.25):
    U = clg.CFieldGaugeSU3(lat)
    if kind == "haar":
        U.InitialField(clg.GAUGE_HAAR, seed, 1)
    else:
        U.InitialField(clg.GAUGE_EXPH, seed, 1, eps)
    return U


def test_generator_matches_oracle(ctx, clg, oracle):
    lat = clg.Lattice(ctx, (4, 4, 4, 8))
    L = lat.dims
    for kind in ("haar", "expH"):
        U = make_gauge(clg, lat, kind, seed=0xC1A60001)
        want = oracle.gauge_haar(L, 0xC1A60001, 1) if kind == "haar" else oracle.gauge_expH(L, 0xC1A60001, 0.25)
        np.testing.assert_allclose(U.CopyDataOut(), want, atol=1e-13)
        assert U.unitarity() < 1e-13
        assert abs(U.plaquette() - oracle.plaquette(L, want)) < 1e-13
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    f.InitialField(clg.SOURCE_GAUSS, 99, 2)
    np.testing.assert_allclose(f.to_numpy(), oracle.gauss(lat.volume, 12, 99, 2).reshape(-1, 4, 3), atol=1e-14)
    f.InitialField(clg.SOURCE_Z2, 98, 3)
    np.testing.assert_array_equal(f.to_numpy(), oracle.z2(lat.volume, 12, 98, 3).reshape(-1, 4, 3))
    f.InitialField(clg.SOURCE_Z4, 97, 4)
    np.testing.assert_array_equal(f.to_numpy(), oracle.z4(lat.volume, 12, 97, 4).reshape(-1, 4, 3))


def test_bridgepp_import_plaquette(ctx, clg):
    """Known answer of TestConfigurationFileIO.cpp:12-38 through the Bridge++ loader."""
    g = np.load(os.path.join(GOLDEN, "bridgepp_4x4x4x8.npz"))
    lat = clg.Lattice(ctx, tuple(int(v) for v in g["dims"]))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialWithByte(g["links"], clg.LAYOUT_BRIDGEPP)
    assert abs(U.plaquette() - 0.625129946974942) < 1e-12


# (6, 10, 14, 12): extents that are not powers of two, for the multiply-high
# division that turns a checkerboard index into coordinates
@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (4, 6, 4, 8), (2, 2, 2, 2), (6, 10, 14, 12)])
@pytest.mark.parametrize("dagger", [False, True])
def test_wilson_D_fp64(ctx, clg, oracle, dims, dagger):
    lat = clg.Lattice(ctx, dims)
    U = make_gauge(clg, lat)
    Uh = U.CopyDataOut()
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    f.InitialField(clg.SOURCE_GAUSS, 5, 2)
    psi = f.to_numpy()
    (f.Ddagger if dagger else f.D)(U)
    want = oracle.wilson_D(dims, Uh, psi, KAPPA, dagger=dagger)
    assert rel(f.to_numpy(), want) < 1e-12


def test_wilson_coefficients_and_products(ctx, clg, oracle, lat8):
    L = lat8.dims
    U = make_gauge(clg, lat8)
    Uh = U.CopyDataOut()
    f = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA)
    f.InitialField(clg.SOURCE_GAUSS, 6, 2)
    psi = f.to_numpy()
    g = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA)
    for ct, c, expect in [(clg.EOCT_Minus, 0, -1.0), (clg.EOCT_Real, 0.7, 0.7), (clg.EOCT_Complex, 0.3, 0.3 - 0.2j)]:
        f.apply_to(clg.EFO_F_D, g, U, ct, c, -0.2)
        assert rel(g.to_numpy(), expect * oracle.wilson_D(L, Uh, psi, KAPPA)) < 1e-12
    f.apply_to(clg.EFO_F_DDdagger, g, U)
    want = oracle.wilson_D(L, Uh, oracle.wilson_D(L, Uh, psi, KAPPA, dagger=True), KAPPA)
    assert rel(g.to_numpy(), want) < 1e-12
    # EFO_F_DD (DDS, CFieldFermionWilsonSquareSU3.cu:989-1014): D applied twice, the coefficient once
    f.apply_to(clg.EFO_F_DD, g, U, clg.EOCT_Real, 0.5)
    want = 0.5 * oracle.wilson_D(L, Uh, oracle.wilson_D(L, Uh, psi, KAPPA), KAPPA)
    assert rel(g.to_numpy(), want) < 1e-12
    # hopping blocks
    pm = clg.eo_parity(L)
    g.Zero()
    f.apply_to(clg.OP_DEO, g, U)
    h = oracle.wilson_hop(L, Uh, psi, 0)
    assert rel(g.to_numpy()[pm == 0], h[pm == 0]) < 1e-12


@pytest.mark.parametrize("dagger", [False, True])
def test_wilson_mee_fp64(ctx, clg, oracle, lat8, dagger):
    L = lat8.dims
    U = make_gauge(clg, lat8, "expH", 0xC1A60001)
    Uh = U.CopyDataOut()
    f = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA, subset=clg.EVEN)
    f.InitialField(clg.SOURCE_GAUSS, 7, 2)
    psi = f.to_numpy()
    pm = clg.eo_parity(L)
    assert np.all(psi[pm == 1] == 0)
    f.ApplyOperator(clg.OP_MEE_DAG if dagger else clg.OP_MEE, U)
    want = oracle.wilson_mee(L, Uh, psi, KAPPA, dagger=dagger)
    assert rel(f.to_numpy()[pm == 0], want[pm == 0]) < 1e-12


@pytest.mark.parametrize("prec,tol", [(1, 2e-6), (2, 5e-3)])
def test_wilson_low_precision(ctx, clg, oracle, lat8, prec, tol):
    L = lat8.dims
    U = make_gauge(clg, lat8)
    Uh = U.CopyDataOut()
    f = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA, precision=prec)
    f64 = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA)
    f64.InitialField(clg.SOURCE_GAUSS, 8, 2)
    psi = f64.to_numpy()
    f.from_numpy(psi)
    f.D(U)
    assert rel(f.to_numpy(), oracle.wilson_D(L, Uh, psi, KAPPA)) < tol
    e = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA, subset=clg.EVEN, precision=prec)
    e.from_numpy(psi)
    e.ApplyOperator(clg.OP_MEE, U)
    pm = clg.eo_parity(L)
    pe = psi.copy()
    pe[pm == 1] = 0
    assert rel(e.to_numpy()[pm == 0], oracle.wilson_mee(L, Uh, pe, KAPPA)[pm == 0]) < tol


@pytest.mark.parametrize("dagger", [False, True])
def test_staggered_fp64(ctx, clg, oracle, lat8, dagger):
    L = lat8.dims
    m = 0.02
    U = make_gauge(clg, lat8, "expH", 0xC1A60004)
    Uh = U.CopyDataOut()
    f = clg.CFieldFermionKSSU3(lat8, m)
    f.InitialField(clg.SOURCE_GAUSS, 9, 2)
    chi = f.to_numpy()
    (f.Ddagger if dagger else f.D)(U)
    assert rel(f.to_numpy(), oracle.ks_D(L, Uh, chi, m, dagger=dagger)) < 1e-12
    e = clg.CFieldFermionKSSU3(lat8, m, subset=clg.EVEN)
    e.from_numpy(chi)
    ce = e.to_numpy()
    e.ApplyOperator(clg.OP_DDDAG_EE, U)
    pm = clg.eo_parity(L)
    assert rel(e.to_numpy()[pm == 0], oracle.ks_dddag_ee(L, Uh, ce, m)[pm == 0]) < 1e-12
    f32 = clg.CFieldFermionKSSU3(lat8, m, precision=1)
    f32.from_numpy(chi)
    (f32.Ddagger if dagger else f32.D)(U)
    assert rel(f32.to_numpy(), oracle.ks_D(L, Uh, chi, m, dagger=dagger)) < 2e-6


@pytest.mark.parametrize("dagger", [False, True])
def test_staggered_fp16(ctx, clg, oracle, lat8, dagger):
    """The FP16 staggered hop (half2 link products, FP32 accumulation) against
    the FP64 oracle's D, D^+ and (D D^+)_ee, two right-hand sides."""
    L = lat8.dims
    m = 0.02
    U = make_gauge(clg, lat8, "expH", 0xC1A60004)
    Uh = U.CopyDataOut()
    f64 = clg.CFieldFermionKSSU3(lat8, m)
    chis = []
    f = clg.CFieldFermionKSSU3(lat8, m, precision=2, nrhs=2)
    for r in range(2):
        f64.InitialField(clg.SOURCE_GAUSS, 19 + r, 2)
        chis.append(f64.to_numpy())
        f.from_numpy(chis[-1], r)
    (f.Ddagger if dagger else f.D)(U)
    for r in range(2):
        assert rel(f.to_numpy(r), oracle.ks_D(L, Uh, chis[r], m, dagger=dagger)) < 5e-3
    e = clg.CFieldFermionKSSU3(lat8, m, subset=clg.EVEN, precision=2)
    pm = clg.eo_parity(L)
    ce = chis[0].copy()
    ce[pm == 1] = 0
    e.from_numpy(ce)
    e.ApplyOperator(clg.OP_DDDAG_EE, U)
    assert rel(e.to_numpy()[pm == 0], oracle.ks_dddag_ee(L, Uh, ce, m)[pm == 0]) < 5e-3


def test_multi_rhs_matches_single(ctx, clg, lat8):
    U = make_gauge(clg, lat8)
    n = 3
    fb = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA, nrhs=n)
    singles = []
    for r in range(n):
        fb.InitialField(clg.SOURCE_GAUSS, 100 + r, 2, rhs=r)
        s = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA)
        s.InitialField(clg.SOURCE_GAUSS, 100 + r, 2)
        s.D(U)
        singles.append(s.to_numpy())
    fb.D(U)
    for r in range(n):
        np.testing.assert_array_equal(fb.to_numpy(r), singles[r])
    d = fb.Dot(fb)
    assert d.shape == (n,)
    for r in range(n):
        assert abs(d[r] - np.vdot(singles[r], singles[r])) < 1e-9 * abs(d[r])


def test_blas(ctx, clg, oracle, lat8):
    a = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA)
    b = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA)
    a.InitialField(clg.SOURCE_GAUSS, 1, 2)
    b.InitialField(clg.SOURCE_GAUSS, 1, 3)
    A, B = a.to_numpy(), b.to_numpy()
    assert abs(a.Dot(b) - oracle.dot(A, B)) < 1e-12 * abs(oracle.dot(A, B)) + 1e-10
    a.Axpy(0.5 - 0.25j, b)
    np.testing.assert_allclose(a.to_numpy(), A + (0.5 - 0.25j) * B, atol=1e-14)
    a.ScalarMultply(2j)
    np.testing.assert_allclose(a.to_numpy(), 2j * (A + (0.5 - 0.25j) * B), atol=1e-14)
    c = clg.CFieldFermionWilsonSquareSU3(lat8, KAPPA, precision=1)
    b.CopyTo(c)
    np.testing.assert_allclose(c.to_numpy(), B, atol=1e-6)
