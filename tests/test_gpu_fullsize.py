"""Parity at the full sizes the benchmark numbers are quoted on, against the
FP64 oracle.

* 32^3x16 (Wilson, even-odd solves), 48^3x24 (Dslash precisions) and
  32^3x32 (batched point + Z2 sources): the FP64 operator to 1e-12 norm-wise,
  which also covers the 32-bit checkerboard index arithmetic and the
  multiply-high coordinate division at these extents;
* the FP32 and FP16 operators, with their errors against the FP64 oracle
  printed and bounded (2e-6 FP32, 5e-3 FP16 storage, as in the small tests);
* the headline solves (FP16-inner CGNE in FP64 defect correction, and FP32
  inner) with the true relative residual |b - D x| / |b| recomputed by the
  oracle's FP64 operator: <= 1e-10 for every right-hand side;
* staggered (DD^+)_ee at 32^3x16 with 2am = 0.02 and the 12 shifts
  10^(-4 + 5k/11): every shift's true residual by the oracle <= 1e-10.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355
TOL = 1e-10


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def expH(clg, lat, seed):
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, seed, 1, 0.25)
    return U


@pytest.fixture(scope="module")
def c2(ctx, clg, oracle):
    """The single-source 32^3x16 workload: exp(i 0.25 H) links (seed 0xC1A60001), one Gaussian source."""
    lat = clg.Lattice(ctx, (32, 32, 32, 16))
    U = expH(clg, lat, 0xC1A60001)
    Uh = U.CopyDataOut()
    yield lat, U, Uh
    U.close()
    lat.close()


@pytest.mark.parametrize("dagger", [False, True])
def test_config2_wilson_D_fp64(ctx, clg, oracle, c2, dagger):
    lat, U, Uh = c2
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    f.InitialField(clg.SOURCE_GAUSS, 0xC1A60001, 2)
    psi = f.to_numpy()
    (f.Ddagger if dagger else f.D)(U)
    assert rel(f.to_numpy(), oracle.wilson_D(lat.dims, Uh, psi, KAPPA, dagger=dagger)) < 1e-12
    f.close()


def test_config2_mee_all_precisions(ctx, clg, oracle, c2):
    lat, U, Uh = c2
    L = lat.dims
    pm = clg.eo_parity(L)
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN)
    f.InitialField(clg.SOURCE_GAUSS, 0xC1A60001, 2)
    psi = f.to_numpy()
    want = oracle.wilson_mee(L, Uh, psi, KAPPA)[pm == 0]
    errs = {}
    for prec, tol in [(clg.DOUBLE, 1e-12), (clg.SINGLE, 2e-6), (clg.HALF, 5e-3)]:
        e = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=prec)
        e.from_numpy(psi)
        e.ApplyOperator(clg.OP_MEE, U)
        errs[prec] = rel(e.to_numpy()[pm == 0], want)
        e.close()
        assert errs[prec] < tol, (prec, errs[prec])
    print("32^3x16 M_ee error vs FP64 oracle: FP64 %.2e, FP32 %.2e, FP16 %.2e" % (errs[0], errs[1], errs[2]))
    f.close()


@pytest.mark.parametrize("inner", ["half", "single"])
def test_config2_headline_solve(ctx, clg, oracle, c2, inner):
    """D x = b by CGNE on the Schur system, FP16 (headline) or FP32 inner, FP64 outer."""
    lat, U, Uh = c2
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60001, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    S = clg.CSLASolverCG(ctx, inner_precision=clg.HALF if inner == "half" else clg.SINGLE, tol_true_rel=TOL)
    info = S.Solve(x, b, U, clg.EFO_F_D)[0]
    assert info["status"] == 0
    op = oracle.Operator("WILSON_D", lat.dims, Uh, KAPPA)
    r = op.true_residual(b.to_numpy(), x.to_numpy())
    print("32^3x16 %s-inner CGNE: %d applications, oracle true residual %.3e" % (inner, info["iterations"], r))
    assert r <= TOL
    S.close()
    x.close()
    b.close()


def test_config5_staggered_12_shifts(ctx, clg, oracle):
    """The staggered multi-shift workload: staggered (DD^+)_ee + sigma_k on 32^3x16, 2am = 0.02, FP32 CG-M + FP64 refinement."""
    lat = clg.Lattice(ctx, (32, 32, 32, 16))
    m = 0.02
    U = expH(clg, lat, 0xC1A60004)
    b = clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60004, 2)
    shifts = [10 ** (-4 + 5 * k / 11) for k in range(12)]
    xs = [clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN) for _ in shifts]
    S = clg.CMultiShiftCG(ctx, inner_precision=clg.SINGLE)
    infos = S.Solve(xs, shifts, b, U, clg.OP_DDDAG_EE)
    op = oracle.Operator("KS_DDDAG_EE", lat.dims, U.CopyDataOut(), m)
    bh = b.to_numpy()
    worst = 0.0
    for k, s in enumerate(shifts):
        assert infos[k]["status"] == 0
        r = op.true_residual(bh, xs[k].to_numpy(), complex(s))
        worst = max(worst, r)
        assert r <= TOL, (k, s, r)
    print("staggered 32^3x16 CG-M: worst oracle true residual over 12 shifts %.3e" % worst)


def test_config3_operator_and_solve(ctx, clg, oracle):
    """The large 48^3x24 lattice (V = 2,654,208), FP64 M_ee to 1e-12, FP32 / FP16
    errors stated, and an FP16-inner solve to the oracle's true residual 1e-10."""
    lat = clg.Lattice(ctx, (48, 48, 48, 24))
    L = lat.dims
    U = expH(clg, lat, 0xC1A60002)
    Uh = U.CopyDataOut()
    pm = clg.eo_parity(L)
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN)
    f.InitialField(clg.SOURCE_GAUSS, 0xC1A60002, 2)
    psi = f.to_numpy()
    want = oracle.wilson_mee(L, Uh, psi, KAPPA)[pm == 0]
    errs = []
    for prec, tol in [(clg.DOUBLE, 1e-12), (clg.SINGLE, 2e-6), (clg.HALF, 5e-3)]:
        e = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=prec)
        e.from_numpy(psi)
        e.ApplyOperator(clg.OP_MEE, U)
        errs.append(rel(e.to_numpy()[pm == 0], want))
        e.close()
        assert errs[-1] < tol, (prec, errs[-1])
    print("48^3x24 M_ee error vs FP64 oracle: FP64 %.2e, FP32 %.2e, FP16 %.2e" % tuple(errs))
    del want
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60002, 3)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    S = clg.CSLASolverCG(ctx, inner_precision=clg.HALF, tol_true_rel=TOL)
    info = S.Solve(x, b, U, clg.EFO_F_D)[0]
    assert info["status"] == 0
    op = oracle.Operator("WILSON_D", L, Uh, KAPPA)
    r = op.true_residual(b.to_numpy(), x.to_numpy())
    print("48^3x24 FP16-inner CGNE: %d applications, oracle true residual %.3e" % (info["iterations"], r))
    assert r <= TOL


def test_config4_batched_point_and_z2(ctx, clg, oracle):
    """The batched workload's shape: 32^3x32, point sources and Z2 noise in one batched
    FP16-inner solve (a subset of the 28 sources, to keep the oracle's checks short)."""
    lat = clg.Lattice(ctx, (32, 32, 32, 32))
    U = expH(clg, lat, 0xC1A60003)
    n = 4
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    b.InitialAsSource(0, 0, rhs=0)
    b.InitialAsSource(0, 11, rhs=1)
    b.InitialField(clg.SOURCE_Z2, 0xC1A60003, 14, rhs=2)
    b.InitialField(clg.SOURCE_Z2, 0xC1A60003, 15, rhs=3)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    S = clg.CSLASolverCG(ctx, inner_precision=clg.HALF, tol_true_rel=TOL)
    infos = S.Solve(x, b, U, clg.EFO_F_D)
    op = oracle.Operator("WILSON_D", lat.dims, U.CopyDataOut(), KAPPA)
    for r in range(n):
        assert infos[r]["status"] == 0
        res = op.true_residual(b.to_numpy(r), x.to_numpy(r))
        assert res <= TOL, (r, res)
