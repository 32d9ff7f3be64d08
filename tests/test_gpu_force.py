"""HMC fermion forces on the GPU against the FP64 oracle: the Wilson force
(_kernelDWilsonForceSU3, CFieldFermionWilsonSquareSU3.cu:170-231) and its whole
force step (CalculateForceS, :1016-1100: solve, cache, D^+, force), and the
staggered rational force (_kernelDFermionKSForce, CFieldFermionKSSU3.cu:216-262)
with its force step (CalculateForceS, :412-500: multi-shift solve, D0, force)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def setup(clg, ctx, dims, bc, nrhs=1):
    lat = clg.Lattice(ctx, dims, bc)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 0xC1A60031, 1)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_EXPH, 0xC1A60032, 1, 0.3)  # a non-zero start: F is accumulated into
    X = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
    Y = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
    for r in range(nrhs):
        X.InitialField(clg.SOURCE_GAUSS, 0xC1A60033, 2 + r, rhs=r)
        Y.InitialField(clg.SOURCE_GAUSS, 0xC1A60034, 2 + r, rhs=r)
    return lat, U, F, X, Y


@pytest.mark.parametrize("dims,bc", [((8, 8, 8, 8), (1, 1, 1, -1)), ((4, 6, 8, 4), (1, 1, 1, -1)),
                                     ((6, 4, 4, 8), (-1, 1, -1, 1))])
def test_wilson_force_matches_oracle(ctx, clg, oracle, dims, bc):
    """F += force(U, X, Y) on arbitrary X, Y (the kernel is bilinear in them),
    uneven extents and boundary signs in several directions: FP64 parity 1e-12."""
    lat, U, F, X, Y = setup(clg, ctx, dims, bc)
    Uh, F0, Xh, Yh = U.CopyDataOut(), F.CopyDataOut(), X.to_numpy(), Y.to_numpy()
    clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(F, Y, X, U)
    want = oracle.wilson_force(dims, Uh, Xh, Yh, KAPPA, F=F0, bc=bc)
    got = F.CopyDataOut()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want - F0).max()
    # the added part is traceless anti-hermitian
    d = got - F0
    assert np.abs(d + np.conj(np.transpose(d, (0, 2, 1)))).max() < 1e-13 * np.abs(d).max()


def test_wilson_force_sums_right_hand_sides(ctx, clg, oracle):
    """A field of several right-hand sides (pseudofermions) adds each one's force."""
    dims = (4, 4, 8, 8)
    lat, U, F, X, Y = setup(clg, ctx, dims, (1, 1, 1, -1), nrhs=3)
    Uh, want = U.CopyDataOut(), F.CopyDataOut()
    for r in range(3):
        want = oracle.wilson_force(dims, Uh, X.to_numpy(r), Y.to_numpy(r), KAPPA, F=want)
    clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(F, Y, X, U)
    assert rel(F.CopyDataOut(), want) < 1e-13


def test_wilson_force_rejects_bad_arguments(ctx, clg):
    lat, U, F, X, Y = setup(clg, ctx, (4, 4, 4, 4), (1, 1, 1, -1))
    with pytest.raises(clg.CLGError):
        clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(U, Y, X, U)  # F is the gauge field
    Xs = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, precision=clg.SINGLE)
    with pytest.raises(clg.CLGError):
        clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(F, Y, Xs, U)
    Xe = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN)
    with pytest.raises(clg.CLGError):
        clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(F, Y, Xe, U)


@pytest.mark.parametrize("prec", [0, 2])
def test_calculate_force_end_to_end(ctx, clg, oracle, prec):
    """CalculateForceS: D D^+ X = phi solved to 1e-10 (FP64 and FP16-inner CG),
    X cached, Y = D^+ X, F += force.  Against the oracle's force of its own FP64
    CG solution; the second call starts from the cache and needs far fewer
    operator applications."""
    dims = (8, 8, 8, 8)
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60035, 1, 0.25)
    Uh = U.CopyDataOut()
    phi = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    phi.InitialField(clg.SOURCE_GAUSS, 0xC1A60036, 2)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_ZERO)
    cache = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    cache.Zero()
    S = clg.CSLASolverCG(ctx, inner_precision=prec)
    info1 = phi.CalculateForceS(U, F, S, cache)[0]
    assert info1["status"] == 0 and info1["true_rel_residual"] <= 1e-10

    op = oracle.Operator("WILSON_DDDAG", dims, Uh, KAPPA)
    Xo, io = oracle.cg(op, phi.to_numpy(), tol=1e-13, maxiter=20000)
    assert io["true_rel_residual"] < 1e-12
    Yo = oracle.wilson_D(dims, Uh, Xo, KAPPA, dagger=True)
    Fo = oracle.wilson_force(dims, Uh, Xo, Yo, KAPPA)
    assert rel(cache.to_numpy(), Xo) < 1e-8
    assert rel(F.CopyDataOut(), Fo) < 1e-8

    info2 = phi.CalculateForceS(U, F, S, cache)[0]
    assert info2["status"] == 0 and info2["true_rel_residual"] <= 1e-10
    assert info2["iterations"] < info1["iterations"] // 4, (info1, info2)
    assert rel(F.CopyDataOut(), 2 * Fo) < 1e-8


@pytest.mark.parametrize("dims,bc,n", [((8, 8, 8, 8), (1, 1, 1, -1), 3), ((4, 6, 8, 4), (-1, 1, 1, -1), 1),
                                       ((6, 4, 4, 8), (1, -1, 1, 1), 7)])
def test_ks_force_matches_oracle(ctx, clg, oracle, dims, bc, n):
    """F -= staggered rational force of arbitrary phi_i, phi_id (the kernel is
    bilinear in them) with n poles, uneven extents and boundary signs: FP64 parity 1e-12."""
    lat = clg.Lattice(ctx, dims, bc)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 0xC1A60051, 1)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_EXPH, 0xC1A60052, 1, 0.3)
    pi = [clg.CFieldFermionKSSU3(lat, 0.1) for _ in range(n)]
    pd = [clg.CFieldFermionKSSU3(lat, 0.1) for _ in range(n)]
    for k in range(n):
        pi[k].InitialField(clg.SOURCE_GAUSS, 0xC1A60053, 2 + k)
        pd[k].InitialField(clg.SOURCE_GAUSS, 0xC1A60054, 2 + k)
    a = np.linspace(0.2, 1.7, n)
    Uh, F0 = U.CopyDataOut(), F.CopyDataOut()
    clg.CFieldFermionKSSU3.DerivateD0(F, U, pi, pd, a)
    want = oracle.ks_force(dims, Uh, [f.to_numpy() for f in pi], [f.to_numpy() for f in pd], a, F=F0, bc=bc)
    got = F.CopyDataOut()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want - F0).max()


def test_ks_force_rejects_bad_arguments(ctx, clg):
    lat = clg.Lattice(ctx, (4, 4, 4, 4))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_IDENTITY)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_ZERO)
    good = clg.CFieldFermionKSSU3(lat, 0.1)
    with pytest.raises(clg.CLGError):
        clg.CFieldFermionKSSU3.DerivateD0(F, U, [], [], [])  # no poles
    with pytest.raises(clg.CLGError):
        clg.CFieldFermionKSSU3.DerivateD0(F, U, [good] * 65, [good] * 65, [1.0] * 65)  # above 64
    even = clg.CFieldFermionKSSU3(lat, 0.1, subset=clg.EVEN)
    with pytest.raises(clg.CLGError):
        clg.CFieldFermionKSSU3.DerivateD0(F, U, [even], [good], [1.0])
    w = clg.CFieldFermionWilsonSquareSU3(lat, 0.1)
    with pytest.raises(clg.CLGError):
        clg.CFieldFermionKSSU3.DerivateD0(F, U, [w], [good], [1.0])


@pytest.mark.parametrize("prec", [0, 1])
def test_ks_calculate_force_end_to_end(ctx, clg, oracle, prec):
    """CalculateForceS for staggered fermions: one multi-shift CG solve of
    (DD^+ + b_i) phi_i = phi (every pole to 1e-10), phi_id = D0 phi_i, F -= force;
    against the oracle's force of its own FP64 multi-shift solutions."""
    dims = (8, 8, 8, 8)
    m = 0.1
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60055, 1, 0.25)
    Uh = U.CopyDataOut()
    phi = clg.CFieldFermionKSSU3(lat, m)
    phi.InitialField(clg.SOURCE_GAUSS, 0xC1A60056, 2)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_ZERO)
    a = [0.05, 0.2, 0.7, 2.5]
    b = [0.002, 0.03, 0.4, 5.0]
    S = clg.CMultiShiftCG(ctx, inner_precision=prec)
    infos = phi.CalculateForceS(U, F, S, a, b)
    assert len(infos) == 4 and all(i["status"] == 0 and i["true_rel_residual"] <= 1e-10 for i in infos), infos
    op = oracle.Operator("KS_DDDAG", dims, Uh, m)
    xs, io = oracle.cgm(op, phi.to_numpy(), b, tol=1e-13)
    Fo = oracle.ks_force(dims, Uh, xs, [oracle.ks_D(dims, Uh, x, 0.0) for x in xs], a)
    assert np.linalg.norm(F.CopyDataOut() - Fo) / np.linalg.norm(Fo) < 1e-8
