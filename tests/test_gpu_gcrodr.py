"""GCRO-DR (CSolverGCRODR.cpp) on the GPU: every solve to the FP64 true relative
residual 1e-10 and equal to the oracle's FP64 GMRES solution; the recycled
subspace kept between solves of one operator cuts the operator applications
of the later solves (the reason the reference has the solver)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355
TOL = 1e-10


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_gcrodr_wilson_full_matches_oracle(ctx, clg, oracle):
    dims = (8, 8, 8, 8)
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60091, 1, 0.25)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60092, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    S = clg.CSLASolverGCRODR(ctx, MDim=20, KDim=8)
    info = S.Solve(x, b, U, clg.EFO_F_D)[0]
    op = oracle.Operator("WILSON_D", dims, U.CopyDataOut(), KAPPA)
    bh, xh = b.to_numpy(), x.to_numpy()
    assert info["status"] == 0 and info["true_rel_residual"] <= TOL
    assert op.true_residual(bh, xh) <= TOL
    xo, _ = oracle.gmres(op, bh, maxdim=12, restart=400, accuracy=1e-26)
    assert rel(xh, xo) < 1e-8


def test_gcrodr_recycling_cuts_applications(ctx, clg, oracle):
    """A sequence of right-hand sides of one near-critical operator (8^4,
    exp(0.1 i H) links, kappa = 0.124: a few isolated low modes), as in an HMC
    trajectory: every solve to 1e-10; the solves after the first start from the
    kept U_k and need far fewer applications than restarted GMRES with the same
    number of new Krylov vectors per cycle (m - k = 8).  Then D^+ and the
    staggered even-odd operator through the same solver."""
    dims = (8, 8, 8, 8)
    kappa = 0.124
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60093, 1, 0.1)
    Uh = U.CopyDataOut()
    S = clg.CSLASolverGCRODR(ctx, MDim=32, KDim=24, Restart=2000)
    op = oracle.Operator("WILSON_D", dims, Uh, kappa)
    apps = []
    for r in range(4):
        b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
        b.InitialField(clg.SOURCE_GAUSS, 0xC1A60094, 2 + r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
        info = S.Solve(x, b, U, clg.EFO_F_D)[0]
        assert info["status"] == 0 and op.true_residual(b.to_numpy(), x.to_numpy()) <= TOL
        apps.append(info["iterations"])
    # restarted GMRES(8) on the same (full, not even-odd reduced) operator
    g8 = clg.CSLASolverGMRES(ctx, MaxDim=8, inner_precision=clg.DOUBLE, even_odd=0)
    gi = g8.Solve(x, b, U, clg.EFO_F_D)[0]
    assert gi["status"] == 0
    assert max(apps[1:]) < 0.75 * gi["iterations"], (apps, gi["iterations"])
    S.Reset()
    info = S.Solve(x, b, U, clg.EFO_F_D)[0]
    assert info["status"] == 0 and info["restarts"] >= 1
    # D^+ through the same solver (a new operator rebuilds the workspace)
    info = S.Solve(x, b, U, clg.EFO_F_Ddagger)[0]
    opd = oracle.Operator("WILSON_DDAG", dims, Uh, kappa)
    assert info["status"] == 0 and opd.true_residual(b.to_numpy(), x.to_numpy()) <= TOL
    # staggered (DD^+)_ee on even fields
    m = 0.05
    be = clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN)
    be.InitialField(clg.SOURCE_GAUSS, 0xC1A60095, 2)
    xe = clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN)
    info = S.Solve(xe, be, U, clg.OP_DDDAG_EE)[0]
    ops = oracle.Operator("KS_DDDAG_EE", dims, Uh, m)
    assert info["status"] == 0 and ops.true_residual(be.to_numpy(), xe.to_numpy()) <= TOL


@pytest.mark.parametrize("space", ["EEDT_REV", "EEDT_HEV"])
def test_gcrodr_deflation_spaces(ctx, clg, oracle, space):
    """DeflateSpace REV (Ritz vectors) and HEV (harmonic Ritz vectors) on the
    near-critical operator: the first solve (one GMRES cycle, FindPk1) and the
    recycled solves after it (FindPk2 every cycle) reach 1e-10 and equal the
    oracle's FP64 GMRES solution."""
    dims = (8, 8, 8, 8)
    kappa = 0.124
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60093, 1, 0.1)
    op = oracle.Operator("WILSON_D", dims, U.CopyDataOut(), kappa)
    S = clg.CSLASolverGCRODR(ctx, MDim=32, KDim=24, Restart=2000, DeflateSpace=getattr(clg, space))
    for r in range(3):
        b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
        b.InitialField(clg.SOURCE_GAUSS, 0xC1A60096, 2 + r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
        info = S.Solve(x, b, U, clg.EFO_F_D)[0]
        bh, xh = b.to_numpy(), x.to_numpy()
        assert info["status"] == 0 and op.true_residual(bh, xh) <= TOL, (space, r, info)
        if r == 2:
            xo, _ = oracle.gmres(op, bh, maxdim=12, restart=2000, accuracy=1e-26)
            assert rel(xh, xo) < 1e-7
    S.close()


def test_gcrodr_rejects_bad_arguments(ctx, clg):
    lat = clg.Lattice(ctx, (4, 4, 4, 4))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 1, 1)
    with pytest.raises(clg.CLGError):
        clg.CSLASolverGCRODR(ctx, MDim=40)
    with pytest.raises(clg.CLGError):
        clg.CSLASolverGCRODR(ctx, MDim=10, KDim=9)
    with pytest.raises(clg.CLGError):
        clg.CSLASolverGCRODR(ctx, DeflateSpace=3)
    S = clg.CSLASolverGCRODR(ctx)
    b2 = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=2)
    x2 = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=2)
    with pytest.raises(clg.CLGError):
        S.Solve(x2, b2, U, clg.EFO_F_D)
    bs = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, precision=clg.SINGLE)
    xs = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, precision=clg.SINGLE)
    with pytest.raises(clg.CLGError):
        S.Solve(xs, bs, U, clg.EFO_F_D)


@pytest.mark.parametrize("space", ["EEDT_SVD", "EEDT_REV", "EEDT_HEV"])
def test_gmres_mdr_recycles(ctx, clg, oracle, space):
    """GMRES-MDR (CSolverGMRESMDR.cpp:16-170): the solves after the first start
    by rotating the kept U_k to the eigenvectors of the deflation type's k x k
    problem (with C_k = A U_k orthonormal again); every solve to the FP64 true
    residual 1e-10, equal to the oracle's GMRES solution, and the recycled solves
    as cheap as GCRO-DR's on the same sequence (the same subspace, another basis)."""
    dims = (8, 8, 8, 8)
    kappa = 0.124
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60093, 1, 0.1)
    Uh = U.CopyDataOut()
    op = oracle.Operator("WILSON_D", dims, Uh, kappa)
    apps = {}
    for name, cls in (("mdr", clg.CSLASolverGMRESMDR), ("gcrodr", clg.CSLASolverGCRODR)):
        S = cls(ctx, MDim=32, KDim=24, Restart=2000, DeflateSpace=getattr(clg, space))
        apps[name] = []
        for r in range(3):
            b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
            b.InitialField(clg.SOURCE_GAUSS, 0xC1A60094, 2 + r)
            x = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
            info = S.Solve(x, b, U, clg.EFO_F_D)[0]
            bh, xh = b.to_numpy(), x.to_numpy()
            assert info["status"] == 0 and op.true_residual(bh, xh) <= TOL
            if name == "mdr" and r == 2:
                xo, _ = oracle.gmres(op, bh, maxdim=12, restart=400, accuracy=1e-26)
                assert rel(xh, xo) < 1e-8
            apps[name].append(info["iterations"])
        S.close()
    assert apps["mdr"][0] == apps["gcrodr"][0]  # the first solve is the same GMRES cycle
    assert max(apps["mdr"][1:]) <= 1.25 * max(apps["gcrodr"][1:]), apps
