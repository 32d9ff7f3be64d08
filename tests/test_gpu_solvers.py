"""Solver parity on the GPU: every solve must reach the FP64 true relative
residual 1e-10 (recomputed here by the FP64 oracle) and agree with the oracle's
own FP64 solve; the reference's solver identities (Tests/TestSolver.cpp:12-120)
are checked at that tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355
TOL = 1e-10


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def gauge(clg, lat, kind, seed):
    U = clg.CFieldGaugeSU3(lat)
    if kind == "haar":
        U.InitialField(clg.GAUGE_HAAR, seed, 1)
    else:
        U.InitialField(clg.GAUGE_EXPH, seed, 1, 0.25)
    return U


@pytest.mark.parametrize("solver,prec", [("GMRES", 0), ("BiCGStab", 0), ("GMRES", 1), ("BiCGStab", 1), ("BiCGStab", 2),
                                         ("GMRES", 2)])
def test_wilson_solve_haar_8x4(ctx, clg, oracle, solver, prec):
    """8^4 Haar links, kappa 0.1355, Gaussian source, D x = b."""
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    U = gauge(clg, lat, "haar", 0xC1A60000)
    Uh = U.CopyDataOut()
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60000, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    S = (clg.CSLASolverGMRES if solver == "GMRES" else clg.CSLASolverBiCGStab)(ctx, inner_precision=prec)
    info = S.Solve(x, b, U, clg.EFO_F_D)[0]
    op = oracle.Operator("WILSON_D", lat.dims, Uh, KAPPA)
    bh, xh = b.to_numpy(), x.to_numpy()
    assert info["status"] == 0
    assert op.true_residual(bh, xh) <= TOL
    assert info["true_rel_residual"] <= TOL
    xo, io = oracle.gmres(op, bh, maxdim=12, restart=200, accuracy=1e-24)
    assert rel(xh, xo) < 1e-8


def test_wilson_inverse_identities(ctx, clg, oracle):
    """|D^-1 D phi - phi|, |D D^-1 phi - phi| and the D^+ / DD^+ forms (TestSolver.cpp:12-120)."""
    lat = clg.Lattice(ctx, (4, 4, 4, 8))
    U = gauge(clg, lat, "haar", 17)
    phi = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    phi.InitialField(clg.SOURCE_GAUSS, 18, 2)
    ph = phi.to_numpy()
    S = clg.CSLASolverGMRES(ctx, inner_precision=1)
    for op, apply in [(clg.EFO_F_D, "D"), (clg.EFO_F_Ddagger, "Ddagger"), (clg.EFO_F_DDdagger, "DDdagger")]:
        y = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
        phi.CopyTo(y)
        getattr(y, apply)(U)
        x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
        S.Solve(x, y, U, op)  # D^-1 D phi
        assert rel(x.to_numpy(), ph) < 1e-8
        z = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
        S.Solve(z, phi, U, op)  # D D^-1 phi
        getattr(z, apply)(U)
        assert rel(z.to_numpy(), ph) <= TOL


@pytest.mark.parametrize("solver", ["GMRES", "BiCGStab"])
def test_wilson_near_critical_small(ctx, clg, oracle, solver):
    """exp(i eps H) links at eps = 0.25, kappa = 0.1355 (near-critical) on 4^3 x 8."""
    lat = clg.Lattice(ctx, (4, 4, 4, 8))
    U = gauge(clg, lat, "expH", 0xC1A60001)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    b.InitialField(clg.SOURCE_GAUSS, 3, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    S = (clg.CSLASolverGMRES if solver == "GMRES" else clg.CSLASolverBiCGStab)(ctx, inner_precision=1)
    info = S.Solve(x, b, U, clg.EFO_F_D)[0]
    op = oracle.Operator("WILSON_D", lat.dims, U.CopyDataOut(), KAPPA)
    assert op.true_residual(b.to_numpy(), x.to_numpy()) <= TOL
    assert info["status"] == 0


def test_wilson_schur_system_direct(ctx, clg, oracle):
    """Solve M_ee x_e = b_e directly on EVEN fields."""
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    U = gauge(clg, lat, "expH", 0xC1A60001)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN)
    b.InitialField(clg.SOURCE_GAUSS, 4, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN)
    S = clg.CSLASolverBiCGStab(ctx, inner_precision=1)
    info = S.Solve(x, b, U, clg.OP_MEE)[0]
    op = oracle.Operator("WILSON_MEE", lat.dims, U.CopyDataOut(), KAPPA)
    assert op.true_residual(b.to_numpy(), x.to_numpy()) <= TOL
    assert info["iterations"] > 0


def test_multi_rhs_batch(ctx, clg, oracle):
    """12 spin-colour point sources + Z2 noise sources solved in one batched call."""
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    U = gauge(clg, lat, "expH", 0xC1A60003)
    n = 14
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    for r in range(12):
        b.InitialAsSource(0, r, rhs=r)
    for r in range(12, n):
        b.InitialField(clg.SOURCE_Z2, 0xC1A60003, 10 + r, rhs=r)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    S = clg.CSLASolverBiCGStab(ctx, inner_precision=1)
    infos = S.Solve(x, b, U, clg.EFO_F_D)
    op = oracle.Operator("WILSON_D", lat.dims, U.CopyDataOut(), KAPPA)
    for r in range(n):
        assert infos[r]["status"] == 0
        assert op.true_residual(b.to_numpy(r), x.to_numpy(r)) <= TOL


@pytest.mark.parametrize("op,name", [(0, "WILSON_D"), (1, "WILSON_DDAG")])
@pytest.mark.parametrize("prec", [1, 2])
def test_wilson_cg_normal_equations(ctx, clg, oracle, op, name, prec):
    """CG on a Wilson D (D^+) solve runs CGNE (CGNR) on the even-odd Schur system."""
    lat = clg.Lattice(ctx, (8, 8, 8, 16))
    U = gauge(clg, lat, "expH", 0xC1A60001)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    b.InitialField(clg.SOURCE_GAUSS, 6, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    info = clg.CSLASolverCG(ctx, inner_precision=prec).Solve(x, b, U, op)[0]
    o = oracle.Operator(name, lat.dims, U.CopyDataOut(), KAPPA)
    assert info["status"] == 0
    assert o.true_residual(b.to_numpy(), x.to_numpy()) <= TOL


@pytest.mark.parametrize("prec", [1, 2])
def test_cg_device_loop(clg, oracle, prec, monkeypatch):
    """CG inner solves looping on the device (CLG_DEVICE_LOOP=1: a CUDA-graph
    WHILE node around each chunk with the stop rules evaluated by a kernel)
    against the host-driven chunk loop: same residual bound, same iteration
    counts (the stop rules are the same), two solves in a row (the second
    replays the cached loop graph)."""
    results = {}
    for loop in ("1", "0"):
        monkeypatch.setenv("CLG_DEVICE_LOOP", loop)
        c = clg.Context(0)
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = gauge(clg, lat, "expH", 0xC1A60001)
        b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=2)
        for r in range(2):
            b.InitialField(clg.SOURCE_GAUSS, 26 + r, 2, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=2)
        S = clg.CSLASolverCG(c, inner_precision=prec)
        o = oracle.Operator("WILSON_D", lat.dims, U.CopyDataOut(), KAPPA)
        for _ in range(2):
            infos = S.Solve(x, b, U, clg.EFO_F_D)
            for r in range(2):
                assert infos[r]["status"] == 0
                assert o.true_residual(b.to_numpy(r), x.to_numpy(r)) <= TOL
        results[loop] = [i["iterations"] for i in infos]
        S.close()
        c.close()
    assert results["1"] == results["0"]


@pytest.mark.parametrize("op,name", [(0, "WILSON_D"), (1, "WILSON_DDAG")])
@pytest.mark.parametrize("prec", [0, 1, 2])
def test_wilson_cg_fused_matches_unfused(clg, oracle, op, name, prec, monkeypatch):
    """The CG iteration whose vector updates run in the Schur hops' epilogues
    (the default) against the one with separate (p, Ap) / update kernels
    (CLG_FUSED_CG=0): both reach the FP64 true residual, on two right-hand
    sides, with iteration counts that agree to within a few percent (they
    differ only in rounding: the fused form never stores A p)."""
    infos, sols = {}, {}
    for fused in ("1", "0"):
        monkeypatch.setenv("CLG_FUSED_CG", fused)
        c = clg.Context(0)
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = gauge(clg, lat, "expH", 0xC1A60001)
        b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=2)
        for r in range(2):
            b.InitialField(clg.SOURCE_GAUSS, 16 + r, 2, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=2)
        infos[fused] = clg.CSLASolverCG(c, inner_precision=prec).Solve(x, b, U, op)
        o = oracle.Operator(name, lat.dims, U.CopyDataOut(), KAPPA)
        for r in range(2):
            assert infos[fused][r]["status"] == 0
            assert o.true_residual(b.to_numpy(r), x.to_numpy(r)) <= TOL
        sols[fused] = [x.to_numpy(r) for r in range(2)]
        c.close()
    for r in range(2):
        n1, n0 = infos["1"][r]["iterations"], infos["0"][r]["iterations"]
        assert abs(n1 - n0) <= max(4, 0.05 * n0), (n1, n0)
        # both solutions have residual <= 1e-10; their distance is bounded by
        # that times the condition number of D
        assert np.linalg.norm(sols["1"][r] - sols["0"][r]) <= 1e-7 * np.linalg.norm(sols["0"][r])


def test_half_precision_point_source(ctx, clg, oracle):
    """A point source makes sites with tiny (float-denormal) maxima after a few
    hops; the FP16 per-site-norm storage must flush them instead of producing NaN."""
    lat = clg.Lattice(ctx, (8, 8, 8, 32))
    U = gauge(clg, lat, "expH", 0xC1A60003)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    b.InitialAsSource(lat.volume // 2 + 3, 0)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    info = clg.CSLASolverCG(ctx, inner_precision=clg.HALF).Solve(x, b, U, clg.EFO_F_D)[0]
    o = oracle.Operator("WILSON_D", lat.dims, U.CopyDataOut(), KAPPA)
    assert info["status"] == 0
    assert o.true_residual(b.to_numpy(), x.to_numpy()) <= TOL
    e = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF)
    e.InitialAsSource(0, 0)
    for _ in range(6):
        e.ApplyOperator(clg.OP_MEE_MEEDAG, U)
    assert np.isfinite(e.to_numpy()).all()


def test_staggered_cg(ctx, clg, oracle):
    """Staggered D x = b through CG on (DD^+)_ee, and DD^+ x = b."""
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    m = 0.02
    U = gauge(clg, lat, "expH", 0xC1A60004)
    b = clg.CFieldFermionKSSU3(lat, m)
    b.InitialField(clg.SOURCE_GAUSS, 5, 2)
    x = clg.CFieldFermionKSSU3(lat, m)
    S = clg.CSLASolverCG(ctx, inner_precision=1)
    S.Solve(x, b, U, clg.EFO_F_D)
    Uh = U.CopyDataOut()
    op = oracle.Operator("KS_D", lat.dims, Uh, m)
    assert op.true_residual(b.to_numpy(), x.to_numpy()) <= TOL
    S.Solve(x, b, U, clg.EFO_F_DDdagger)
    op2 = oracle.Operator("KS_DDDAG", lat.dims, Uh, m)
    assert op2.true_residual(b.to_numpy(), x.to_numpy()) <= TOL


@pytest.mark.parametrize("op", ["D", "Ddagger"])
def test_fused_residual_matches_separate(clg, oracle, op, monkeypatch):
    """The outer residual r = b - D x fused into the FP64 hop's epilogue (with
    |r|^2 and the inner-precision copy) against the separate passes
    (CLG_FUSED_RESID=0): the same outer and inner iteration counts, solutions
    within 1e-9 of each other, both to 1e-10 by the oracle."""
    res = {}
    for fused in ("1", "0"):
        monkeypatch.setenv("CLG_FUSED_RESID", fused)
        c = clg.Context(0)
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = gauge(clg, lat, "expH", 0xC1A60001)
        b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=3)
        for r in range(3):
            b.InitialField(clg.SOURCE_GAUSS, 40 + r, 2, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=3)
        S = clg.CSLASolverCG(c, inner_precision=clg.HALF)
        infos = S.Solve(x, b, U, clg.EFO_F_D if op == "D" else clg.EFO_F_Ddagger)
        o = oracle.Operator("WILSON_D" if op == "D" else "WILSON_DDAG", lat.dims, U.CopyDataOut(), KAPPA)
        for r in range(3):
            assert infos[r]["status"] == 0
            assert o.true_residual(b.to_numpy(r), x.to_numpy(r)) <= TOL
        res[fused] = ([(i["iterations"], i["outer"]) for i in infos], [x.to_numpy(r) for r in range(3)])
        S.close()
        for f in (b, x, U, lat):
            f.close()
        c.close()
    assert res["1"][0] == res["0"][0]
    for r in range(3):
        assert np.linalg.norm(res["1"][1][r] - res["0"][1][r]) <= 1e-9 * np.linalg.norm(res["0"][1][r])
