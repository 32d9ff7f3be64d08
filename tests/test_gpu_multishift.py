"""Multi-shift solves on the GPU: (op + c_n) x_n = b for all n, every shift to
the FP64 true residual 1e-10 (TestMultiShiftSolver.cpp:12-111 identities,
tightened), and the rational-approximation driver (CField.cpp:114-145)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_staggered_cgm_12_shifts(ctx, clg, oracle):
    """The 32^3x16 staggered multi-shift problem on 8^4: (DD^+)_ee + sigma_k, 12 shifts log-spaced 1e-4..10."""
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    m = 0.02
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60004, 1, 0.25)
    b = clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60004, 2)
    shifts = np.logspace(-4, 1, 12)
    xs = [clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN) for _ in shifts]
    S = clg.CMultiShiftCG(ctx, inner_precision=clg.SINGLE)
    infos = S.Solve(xs, list(shifts), b, U, clg.OP_DDDAG_EE)
    op = oracle.Operator("KS_DDDAG_EE", lat.dims, U.CopyDataOut(), m)
    bh = b.to_numpy()
    for k, s in enumerate(shifts):
        assert infos[k]["status"] == 0
        assert op.true_residual(bh, xs[k].to_numpy(), complex(s)) <= TOL


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_staggered_cgm_iterates_like_oracle(ctx, clg, oracle, prec):
    """Multi-shift CG with the shifted x_k, p_k written once per block of
    iterations (coefficients over the block's residuals): every shift at the
    FP64 true residual in every inner precision; in FP64 the shared Krylov
    space takes the oracle's iteration count (same stopping rule) and the
    solutions agree.  12 shifts on 8^3x4 (a solve that ends inside a block)."""
    lat = clg.Lattice(ctx, (8, 8, 8, 4))
    m = 0.02
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60071, 1, 0.25)
    b = clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60072, 2)
    shifts = np.logspace(-3, 1, 12)
    xs = [clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN) for _ in shifts]
    S = clg.CMultiShiftCG(ctx, inner_precision=prec)
    infos = S.Solve(xs, list(shifts), b, U, clg.OP_DDDAG_EE)
    op = oracle.Operator("KS_DDDAG_EE", lat.dims, U.CopyDataOut(), m)
    bh = b.to_numpy()
    for k, s in enumerate(shifts):
        assert infos[k]["status"] == 0
        assert op.true_residual(bh, xs[k].to_numpy(), complex(s)) <= TOL
    if prec == 0:
        xo, io = oracle.cgm(op, bh, list(shifts), tol=0.5 * TOL)
        assert abs(min(i["iterations"] for i in infos) - io["iterations"]) <= 1, (infos, io)
        for k in range(len(shifts)):
            assert np.linalg.norm(xs[k].to_numpy() - xo[k]) <= 1e-9 * np.linalg.norm(xo[k])
    # a second call on the same solver replays the captured iterations
    again = S.Solve(xs, list(shifts), b, U, clg.OP_DDDAG_EE)
    for k, s in enumerate(shifts):
        assert again[k]["status"] == 0
        assert op.true_residual(bh, xs[k].to_numpy(), complex(s)) <= TOL


@pytest.mark.parametrize("prec", [0, 1])
def test_staggered_cgm_fused_matches_unfused(clg, oracle, prec, monkeypatch):
    """Multi-shift CG with (p, A p) reduced in the second hop of the staggered
    Schur operator (the default for FP64 / FP32 iterations) against the separate
    operator and dot passes (CLG_FUSED_CG=0): every shift at the FP64 true
    residual in both, the same iteration count to within one (they differ only
    in the summation order of (p, A p)), solutions within the tolerance."""
    infos, sols = {}, {}
    shifts = list(np.logspace(-3, 1, 8))
    for fused in ("1", "0"):
        monkeypatch.setenv("CLG_FUSED_CG", fused)
        c = clg.Context(0)
        lat = clg.Lattice(c, (8, 8, 8, 8))
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60075, 1, 0.25)
        b = clg.CFieldFermionKSSU3(lat, 0.02, subset=clg.EVEN)
        b.InitialField(clg.SOURCE_GAUSS, 0xC1A60076, 2)
        xs = [clg.CFieldFermionKSSU3(lat, 0.02, subset=clg.EVEN) for _ in shifts]
        S = clg.CMultiShiftCG(c, inner_precision=prec)
        infos[fused] = S.Solve(xs, shifts, b, U, clg.OP_DDDAG_EE)
        op = oracle.Operator("KS_DDDAG_EE", lat.dims, U.CopyDataOut(), 0.02)
        bh = b.to_numpy()
        for k, s in enumerate(shifts):
            assert infos[fused][k]["status"] == 0
            assert op.true_residual(bh, xs[k].to_numpy(), complex(s)) <= TOL
        sols[fused] = [x.to_numpy() for x in xs]
        S.close()
        c.close()
    for k in range(len(shifts)):
        assert abs(infos["1"][k]["iterations"] - infos["0"][k]["iterations"]) <= 1
        assert np.linalg.norm(sols["1"][k] - sols["0"][k]) <= 1e-8 * np.linalg.norm(sols["0"][k])


@pytest.mark.parametrize("prec", [0, 1])
def test_wilson_cgm(ctx, clg, oracle, prec):
    """Multi-shift CG on the Wilson DD^+ (12 spin-colour components: a shorter
    flush block) with 5 shifts, every shift to the FP64 true residual; FP64
    takes the oracle's iteration count."""
    lat = clg.Lattice(ctx, (4, 4, 6, 8))
    kappa = 0.13
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60073, 1, 0.25)
    b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60074, 2)
    shifts = [0.003, 0.05, 0.4, 2.0, 9.0]
    xs = [clg.CFieldFermionWilsonSquareSU3(lat, kappa) for _ in shifts]
    S = clg.CMultiShiftCG(ctx, inner_precision=prec)
    infos = S.Solve(xs, shifts, b, U, clg.EFO_F_DDdagger)
    op = oracle.Operator("WILSON_DDDAG", lat.dims, U.CopyDataOut(), kappa)
    bh = b.to_numpy()
    for k, s in enumerate(shifts):
        assert infos[k]["status"] == 0
        assert op.true_residual(bh, xs[k].to_numpy(), complex(s)) <= TOL
    if prec == 0:
        xo, io = oracle.cgm(op, bh, shifts, tol=0.5 * TOL)
        assert abs(min(i["iterations"] for i in infos) - io["iterations"]) <= 1, (infos, io)
        for k in range(len(shifts)):
            assert np.linalg.norm(xs[k].to_numpy() - xo[k]) <= 1e-9 * np.linalg.norm(xo[k])


@pytest.mark.parametrize("op,name", [("EFO_F_D", "WILSON_D"), ("EFO_F_Ddagger", "WILSON_DDAG"),
                                     ("EFO_F_DDdagger", "WILSON_DDDAG")])
@pytest.mark.parametrize("method", ["FOM", "GMRES", "BiCGStab"])
def test_wilson_fom_ms_complex_shifts(ctx, clg, oracle, op, name, method):
    """CMultiShiftFOM / CMultiShiftBiCGStab over one Krylov space with the reference test's shifts
    {2, 1, 0.5, i, 0.5+0.5i, 1-i} on D, D^+ and DD^+ (TestMultiShiftSolver.cpp:12-111):
    every shift to the FP64 true residual 1e-10, the solutions equal to the
    oracle's restated CMultiShiftFOM, and one shared space (the applications of
    the FOM phase are counted once for all six shifts)."""
    lat = clg.Lattice(ctx, (4, 4, 4, 8))
    kappa = 0.1355
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 21, 1)
    b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    b.InitialField(clg.SOURCE_GAUSS, 22, 2)
    cs = [2, 1, 0.5, 1j, 0.5 + 0.5j, 1 - 1j]
    xs = [clg.CFieldFermionWilsonSquareSU3(lat, kappa) for _ in cs]
    if method == "FOM":
        S = clg.CMultiShiftFOM(ctx, MaxDim=30, Restart=100)
    elif method == "GMRES":  # CMultiShiftGMRES (CMultiShiftGMRES.cpp:113-330)
        S = clg.CMultiShiftGMRES(ctx, MaxDim=10, Restart=200)
    else:  # CMultiShiftBiCGStab (CMultiShiftBiCGStab.cpp:73-437)
        S = clg.CMultiShiftBiCGStab(ctx, DiviationStep=10, MaxStep=100)
    infos = S.Solve(xs, cs, b, U, getattr(clg, op))
    Uh = U.CopyDataOut()
    o = oracle.Operator(name, lat.dims, Uh, kappa)
    bh = b.to_numpy()
    if method == "FOM":
        xo, io = oracle.fom_ms(o, bh, cs, maxdim=30, restart=100, accuracy=1e-12 * np.linalg.norm(bh), absolute=True)
    elif method == "GMRES":
        xo, io = oracle.gmres_ms(o, bh, cs, maxdim=10, restart=200, accuracy=1e-13, absolute=True)
    else:
        xo, io = oracle.bicgstab_ms(o, bh, cs, dev_step=10, max_step=100, accuracy=1e-12)
    for k, c in enumerate(cs):
        assert infos[k]["status"] == 0
        assert o.true_residual(bh, xs[k].to_numpy(), complex(c)) <= TOL
        assert np.linalg.norm(xs[k].to_numpy() - xo[k]) <= 1e-8 * np.linalg.norm(xo[k])
    # one Krylov space: fewer applications than the six separate solves of the
    # nested form need together
    N = clg.CMultiShiftNested(ctx, inner_precision=clg.SINGLE)
    ys = [clg.CFieldFermionWilsonSquareSU3(lat, kappa) for _ in cs]
    ninfo = N.Solve(ys, cs, b, U, getattr(clg, op))
    for k, c in enumerate(cs):
        assert ninfo[k]["status"] == 0
        assert o.true_residual(bh, ys[k].to_numpy(), complex(c)) <= TOL
    assert max(i["iterations"] for i in infos) < sum(i["iterations"] for i in ninfo)


def test_rational_round_trip(ctx, clg, oracle):
    """R_{-1/2}(R_{1/2} phi) ~ phi with the degree-3 coefficients of TestSuit_Solver.yaml:751-754
    is replaced by an exact identity: with a = (1), b = (s), c = 0 the driver returns (A + s)^-1 phi."""
    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    m = 0.1
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 31, 1, 0.25)
    f = clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN)
    f.InitialField(clg.SOURCE_GAUSS, 32, 2)
    phi = f.to_numpy()
    S = clg.CMultiShiftCG(ctx, inner_precision=clg.SINGLE)
    S.rational(f, U, clg.OP_DDDAG_EE, c=0.5, a=[0.25, 2.0], b=[0.1, 1.0])
    op = oracle.Operator("KS_DDDAG_EE", lat.dims, U.CopyDataOut(), m)
    x1, _ = oracle.cgm(op, phi, [0.1, 1.0], tol=1e-12)
    want = 0.5 * phi + 0.25 * x1[0] + 2.0 * x1[1]
    got = f.to_numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-9
