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


def test_wilson_fom_ms_complex_shifts(ctx, clg, oracle):
    """The reference test's shifts {2, 1, 0.5, i, 0.5+0.5i, 1-i} on D (TestMultiShiftSolver.cpp:12-111)."""
    lat = clg.Lattice(ctx, (4, 4, 4, 8))
    kappa = 0.1355
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 21, 1)
    b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    b.InitialField(clg.SOURCE_GAUSS, 22, 2)
    cs = [2, 1, 0.5, 1j, 0.5 + 0.5j, 1 - 1j]
    xs = [clg.CFieldFermionWilsonSquareSU3(lat, kappa) for _ in cs]
    S = clg.CMultiShiftFOM(ctx, inner_precision=clg.SINGLE)
    infos = S.Solve(xs, cs, b, U, clg.EFO_F_D)
    op = oracle.Operator("WILSON_D", lat.dims, U.CopyDataOut(), kappa)
    for k, c in enumerate(cs):
        assert infos[k]["status"] == 0
        assert op.true_residual(b.to_numpy(), xs[k].to_numpy(), complex(c)) <= TOL


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
