"""clg_solve_lattices: right-hand sides on several lattices of uneven volume,
each with its own gauge field, solved in one solve (one kernel per step covers
every lattice).  Every right-hand side must reach the FP64 true residual 1e-10
recomputed by the oracle, and agree with the solve of its lattice alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355
TOL = 1e-10


def build(clg, ctx, dims_list, nrhs_list, seed0=0xC1A60003):
    lats, Us, bs, xs = [], [], [], []
    for i, (dims, n) in enumerate(zip(dims_list, nrhs_list)):
        lat = clg.Lattice(ctx, dims)
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, seed0 + i, 1, 0.25)
        b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
        for r in range(n):
            b.InitialField(clg.SOURCE_GAUSS, seed0 + i, 2 + r, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
        lats.append(lat)
        Us.append(U)
        bs.append(b)
        xs.append(x)
    return lats, Us, bs, xs


@pytest.mark.parametrize("solver,inner,opname", [("CG", "HALF", "EFO_F_D"), ("CG", "SINGLE", "EFO_F_Ddagger"),
                                                  ("GMRES", "SINGLE", "EFO_F_D"), ("BiCGStab", "DOUBLE", "EFO_F_D")])
def test_lattices_match_single_solves(ctx, clg, oracle, solver, inner, opname):
    dims_list = [(4, 4, 4, 4), (6, 6, 6, 8), (8, 8, 8, 8), (4, 6, 8, 10)]
    nrhs_list = [2, 1, 3, 2]
    lats, Us, bs, xs = build(clg, ctx, dims_list, nrhs_list)
    cls = {"CG": clg.CSLASolverCG, "GMRES": clg.CSLASolverGMRES, "BiCGStab": clg.CSLASolverBiCGStab}[solver]
    prec = getattr(clg, inner)
    op = getattr(clg, opname)
    S = cls(ctx, inner_precision=prec, tol_true_rel=TOL)
    infos = S.SolveLattices(xs, bs, Us, op)
    assert len(infos) == sum(nrhs_list)
    k = 0
    for i, dims in enumerate(dims_list):
        name = "WILSON_D" if opname == "EFO_F_D" else "WILSON_DDAG"
        o = oracle.Operator(name, dims, Us[i].CopyDataOut(), KAPPA)
        single = clg.CFieldFermionWilsonSquareSU3(lats[i], KAPPA, nrhs=nrhs_list[i])
        S1 = cls(ctx, inner_precision=prec, tol_true_rel=TOL)
        S1.Solve(single, bs[i], Us[i], op)
        for r in range(nrhs_list[i]):
            assert infos[k]["status"] == 0, infos[k]
            xb = xs[i].to_numpy(r)
            assert o.true_residual(bs[i].to_numpy(r), xb) <= TOL
            xsgl = single.to_numpy(r)
            assert np.linalg.norm(xb - xsgl) <= 1e-8 * np.linalg.norm(xsgl)
            k += 1


def test_uneven_set_of_config4(ctx, clg, oracle):
    """The uneven five-lattice set (8^4, 12^4, 16^4, 16^3x32, 24^3x16),
    4 Gaussian sources each, FP16-inner CGNE, in one solve."""
    dims_list = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (16, 16, 16, 32), (24, 24, 24, 16)]
    lats, Us, bs, xs = build(clg, ctx, dims_list, [4] * 5)
    S = clg.CSLASolverCG(ctx, inner_precision=clg.HALF, tol_true_rel=TOL)
    for _ in range(2):  # the second call reuses the batch and its captured graphs
        infos = S.SolveLattices(xs, bs, Us, clg.EFO_F_D)
    k = 0
    for i, dims in enumerate(dims_list):
        o = oracle.Operator("WILSON_D", dims, Us[i].CopyDataOut(), KAPPA)
        for r in range(4):
            assert infos[k]["status"] == 0
            assert o.true_residual(bs[i].to_numpy(r), xs[i].to_numpy(r)) <= TOL
            k += 1
