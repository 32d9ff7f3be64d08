"""Measurements on top of the batched solves against the FP64 oracle: the meson
correlator of 12 point-source propagators (CMeasureMesonCorrelator.cu) and the
Z4-noise condensate traces (CMeasureChiralCondensate.cu, CMeasurementManager.cpp:71-115)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355


def test_meson_contract_matches_oracle(ctx, clg, oracle):
    """_kernelCalculateCorrelatorSU3 + spatial sums on 12 arbitrary fields, all 24 gammas."""
    dims = (4, 6, 4, 8)
    lat = clg.Lattice(ctx, dims)
    prop = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=12)
    for r in range(12):
        prop.InitialField(clg.SOURCE_GAUSS, 0xC1A60081, 2 + r, rhs=r)
    props = [prop.to_numpy(r) for r in range(12)]
    m = clg.CMeasureMesonCorrelator(None, lat, KAPPA, gammas=clg.GAMMAS)
    got = m.contract(prop)
    for k, name in enumerate(clg.GAMMAS):
        want = oracle.meson_correlator(dims, props, k)
        np.testing.assert_allclose(got[name], want, rtol=1e-12, atol=1e-12 * np.abs(want).max(), err_msg=name)


def test_meson_correlator_end_to_end(ctx, clg, oracle):
    """The 12 point sources at the origin solved in one batched call (mixed
    precision, every rhs to 1e-10), then the correlator for several gammas,
    against the oracle's correlator of its own FP64 solutions."""
    dims = (8, 8, 8, 8)
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60082, 1, 0.25)
    Uh = U.CopyDataOut()
    S = clg.CSLASolverBiCGStab(ctx, inner_precision=clg.SINGLE)
    gammas = ["UNITY", "GAMMA4", "GAMMA5", "GAMMA54", "GAMMA45"]
    m = clg.CMeasureMesonCorrelator(S, lat, KAPPA, gammas=gammas)
    got, infos = m.Calculate(U)
    assert len(infos) == 12 and all(i["status"] == 0 and i["true_rel_residual"] <= 1e-10 for i in infos)
    op = oracle.Operator("WILSON_D", dims, Uh, KAPPA)
    V = lat.volume
    props = []
    for r in range(12):
        src = np.zeros((V, 4, 3), np.complex128)
        src[0, r // 3, r % 3] = 1.0
        x, info = oracle.gmres(op, src, maxdim=12, restart=400, accuracy=1e-26)
        assert info["true_rel_residual"] < 1e-12
        props.append(x)
    for k, name in enumerate(gammas):
        want = oracle.meson_correlator(dims, props, clg.GAMMAS.index(name))
        np.testing.assert_allclose(got[name], want, rtol=1e-8, atol=1e-9 * np.abs(want).max(), err_msg=name)
    # a second configuration enters the running average
    m.Calculate(U)
    assert m.count == 2
    np.testing.assert_allclose(m.results[2], got["GAMMA5"], rtol=1e-9)


def test_condensate_end_to_end(ctx, clg, oracle):
    """Z4 noise vectors (the oracle's Z4 generator, bit for bit), psi = D^-1 eta
    in one batched solve (every rhs to 1e-10), and the nine traces: per rhs
    against the oracle's traces of the same fields, averaged over the noise."""
    dims = (8, 8, 8, 8)
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60083, 1, 0.25)
    S = clg.CSLASolverGMRES(ctx, inner_precision=clg.SINGLE)
    n = 4
    c = clg.CMeasureChiralCondensate(S, lat, KAPPA, fields=n)
    avg, infos = c.Calculate(U, seed=0xC1A60084)
    assert len(infos) == n and all(i["status"] == 0 and i["true_rel_residual"] <= 1e-10 for i in infos)
    op = oracle.Operator("WILSON_D", dims, U.CopyDataOut(), KAPPA)
    per = clg.CMeasureChiralCondensate.contract(c.eta, c.psi)
    want_avg = np.zeros(9, np.complex128)
    for r in range(n):
        eta = c.eta.to_numpy(r)
        np.testing.assert_array_equal(eta, oracle.z4(lat.volume, 12, 0xC1A60084, r + 1).reshape(-1, 4, 3))
        psi = c.psi.to_numpy(r)
        assert op.true_residual(eta, psi) <= 1e-10
        for k in range(9):
            w = oracle.condensate(eta, psi, k)
            assert abs(per[r, k] - w) <= 1e-12 * max(abs(w), 1e-3)
            want_avg[k] += w / n
    np.testing.assert_allclose(avg, want_avg, rtol=1e-12, atol=1e-15)
    # the chiral condensate (kind 0) of Wilson fermions: Re <eta^+ D^-1 eta>/V > 0
    assert avg[0].real > 0
