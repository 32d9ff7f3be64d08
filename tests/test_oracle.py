"""CPU tests of the FP64 oracle: pinned to the reference's known answers and
identities (Code/CLGTest/Tests/*), runnable without a GPU."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

KAPPA = 0.1355


def test_bridgepp_plaquette_known_answer(oracle):
    """TestConfigurationFileIO.cpp:12-38: Bridge++ 4^3x8 plaquette 0.625129946974942."""
    g = np.load(os.path.join(GOLDEN, "bridgepp_4x4x4x8.npz"))
    L = tuple(int(v) for v in g["dims"])
    U = oracle.bridgepp_to_clg(L, g["links"])
    assert abs(oracle.plaquette(L, U) - float(g["plaquette"])) < 1e-12
    assert oracle.unitarity_deviation(U) < 1e-12


def test_gamma_table_matches_reference_source(oracle):
    """The oracle's chiral gamma table equals the one parsed from GammaMatrix.h."""
    ref = json.load(open(os.path.join(GOLDEN, "gamma_chiral.json")))["rows"]
    L = (2, 2, 2, 2)
    # probe the oracle's Wilson hopping with identity links on a point source:
    # H^(+) on a point source at the origin gives (1 -/+ g_mu) psi at the neighbours.
    U = oracle.gauge_identity(L)
    for mu, name in enumerate(["GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4"]):
        G = np.zeros((4, 4), complex)
        for r, (c, b) in enumerate(ref[name]):
            G[r, c] = 1j ** b
        for s in range(4):
            psi = np.zeros((16, 4, 3), complex)
            psi[0, s, 0] = 1.0
            out = oracle.wilson_hop(L, U, psi, out_parity=1, bc=(1, 1, 1, 1))
            # site x - mu of the origin (wraps to coordinate 1 in direction mu):
            # receives (1 - g_mu) U psi(x + mu) from its forward hop plus, since L=2,
            # (1 + g_mu) U^+ psi(x - mu) from its backward hop: total 2 psi.
            # Use the forward/backward split through the dagger operator instead:
            outd = oracle.wilson_hop(L, U, psi, out_parity=1, dagger=True, bc=(1, 1, 1, 1))
            c = [0, 0, 0, 0]
            c[mu] = 1
            site = ((c[0] * 2 + c[1]) * 2 + c[2]) * 2 + c[3]
            e = np.zeros(4, complex)
            e[s] = 1
            np.testing.assert_allclose(out[site, :, 0], 2 * e, atol=1e-14)
            np.testing.assert_allclose(outd[site, :, 0], 2 * e, atol=1e-14)
    # on L=4 the forward and backward hops land on different sites
    L = (4, 4, 4, 4)
    U = oracle.gauge_identity(L)
    for mu, name in enumerate(["GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4"]):
        G = np.zeros((4, 4), complex)
        for r, (c, b) in enumerate(ref[name]):
            G[r, c] = 1j ** b
        for s in range(4):
            psi = np.zeros((256, 4, 3), complex)
            psi[0, s, 0] = 1.0
            out = oracle.wilson_hop(L, U, psi, out_parity=1, bc=(1, 1, 1, 1))
            c = [0, 0, 0, 0]
            c[mu] = 3  # x - mu of the origin: its forward hop reaches the origin
            site = ((c[0] * 4 + c[1]) * 4 + c[2]) * 4 + c[3]
            e = np.zeros(4, complex)
            e[s] = 1
            np.testing.assert_allclose(out[site, :, 0], (np.eye(4) - G) @ e, atol=1e-14)
            c[mu] = 1  # x + mu: its backward hop reaches the origin
            site = ((c[0] * 4 + c[1]) * 4 + c[2]) * 4 + c[3]
            np.testing.assert_allclose(out[site, :, 0], (np.eye(4) + G) @ e, atol=1e-14)


def test_philox_known_answers(oracle):
    """Philox4x32-10 known-answer vectors of the Random123 distribution (Salmon et al., SC'11)."""
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in kat:
        assert tuple(int(v) for v in oracle.philox(ctr, key)) == want


def test_generators(oracle):
    L = (4, 4, 4, 4)
    U = oracle.gauge_haar(L, 0xC1A60000, 1)
    assert oracle.unitarity_deviation(U) < 1e-13
    Ue = oracle.gauge_expH(L, 0xC1A60001, 0.25)
    assert oracle.unitarity_deviation(Ue) < 1e-13
    assert 0.7 < oracle.plaquette(L, Ue) < 0.95
    g = oracle.gauss(20000, 12, 7, 2)
    assert abs(np.mean(np.abs(g) ** 2) - 1.0) < 0.02
    z = oracle.z2(1000, 12, 7, 3)
    np.testing.assert_allclose(np.abs(z), 1.0, atol=1e-15)
    z4 = oracle.z4(4000, 12, 7, 3)
    assert set(np.unique(z4).tolist()) == {1, 1j, -1, -1j}
    assert abs(np.mean(z4 == 1j) - 0.25) < 0.01 and abs(np.mean(z4)) < 0.02


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (4, 2, 4, 6)])
def test_wilson_identities(oracle, L):
    """Adjointness <f2, D f1> = <D^+ f2, f1> (Tests/TestCommon.cpp:14-85) and
    gamma5-hermiticity (CFieldFermionWilsonSquareSU3.cu:1362-1500), tightened to FP64."""
    V = oracle.volume(L)
    U = oracle.gauge_haar(L, 11, 1)
    f1 = oracle.gauss(V, 12, 12, 2).reshape(V, 4, 3)
    f2 = oracle.gauss(V, 12, 12, 3).reshape(V, 4, 3)
    d1 = oracle.wilson_D(L, U, f1, KAPPA)
    d2 = oracle.wilson_D(L, U, f2, KAPPA, dagger=True)
    assert abs(oracle.dot(f2, d1) - oracle.dot(d2, f1)) < 1e-12 * V
    g5 = np.array([1, 1, -1, -1])[None, :, None]
    np.testing.assert_allclose(oracle.wilson_D(L, U, f1, KAPPA, dagger=True),
                               g5 * oracle.wilson_D(L, U, g5 * f1, KAPPA), atol=1e-13)
    # D = 1 - kappa (H_e + H_o) and the even-odd Schur identity
    He = oracle.wilson_hop(L, U, f1, 0)
    Ho = oracle.wilson_hop(L, U, f1, 1)
    np.testing.assert_allclose(d1, f1 - KAPPA * (He + Ho), atol=1e-13)


def test_wilson_free_field_plane_wave(oracle):
    """Free field (U = 1, periodic): D e^{ipx} u = [1 - 2 kappa sum cos p_mu + 2 i kappa sum g_mu sin p_mu] e^{ipx} u."""
    L = (4, 4, 4, 8)
    V = oracle.volume(L)
    ref = json.load(open(os.path.join(GOLDEN, "gamma_chiral.json")))["rows"]
    G = []
    for name in ["GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4"]:
        M = np.zeros((4, 4), complex)
        for r, (c, b) in enumerate(ref[name]):
            M[r, c] = 1j ** b
        G.append(M)
    U = oracle.gauge_identity(L)
    x = oracle.coords(L)
    n = np.array([1, 2, 3, 5])
    p = 2 * np.pi * n / np.array(L)
    phase = np.exp(1j * (x @ p))
    u = np.array([0.3 + 0.1j, -0.2j, 0.5, 0.25 - 0.4j])
    col = np.array([1.0, 0.5j, -0.25])
    psi = phase[:, None, None] * u[None, :, None] * col[None, None, :]
    out = oracle.wilson_D(L, U, psi, KAPPA, bc=(1, 1, 1, 1))
    M = (1 - 2 * KAPPA * np.sum(np.cos(p))) * np.eye(4) + 2j * KAPPA * sum(G[m] * np.sin(p[m]) for m in range(4))
    want = phase[:, None, None] * (M @ u)[None, :, None] * col[None, None, :]
    np.testing.assert_allclose(out, want, atol=1e-13)


def test_staggered_antihermitian(oracle):
    """CFieldFermionKSSU3.cu:1424-1491: D_KS(m=0) is anti-Hermitian; D^+ = 2am - H."""
    L = (4, 4, 4, 4)
    V = oracle.volume(L)
    U = oracle.gauge_haar(L, 5, 1)
    a = oracle.gauss(V, 3, 6, 2)
    b = oracle.gauss(V, 3, 6, 3)
    m = 0.02
    assert abs(oracle.dot(b, oracle.ks_D(L, U, a, m)) - oracle.dot(oracle.ks_D(L, U, b, m, dagger=True), a)) < 1e-12
    h = oracle.ks_D(L, U, a, 0.0)
    assert abs(oracle.dot(a, h).real) < 1e-12
    # (D D^+)_ee = m^2 - H_eo H_oe on even sites
    pm = oracle.parity_mask(L)
    ae = a.copy()
    ae[pm == 1] = 0
    full = oracle.ks_D(L, U, oracle.ks_D(L, U, ae, m, dagger=True), m)
    np.testing.assert_allclose(oracle.ks_dddag_ee(L, U, ae, m)[pm == 0], full[pm == 0], atol=1e-13)


def test_oracle_solvers_small(oracle):
    """|D^-1 D phi - phi| (Tests/TestSolver.cpp:12-120) with the FP64 GMRES / BiCGStab restatements."""
    L = (4, 4, 4, 4)
    V = oracle.volume(L)
    U = oracle.gauge_haar(L, 3, 1)
    b = oracle.gauss(V, 12, 4, 2).reshape(V, 4, 3)
    op = oracle.Operator("WILSON_D", L, U, KAPPA)
    x, info = oracle.gmres(op, b, maxdim=12, restart=50, accuracy=1e-24)
    assert info["converged"] and info["true_rel_residual"] < 1e-11
    x2, info2 = oracle.bicgstab(op, b, accuracy=1e-24, std_omega=True)
    assert info2["true_rel_residual"] < 1e-10
    assert np.linalg.norm(x2 - x) / np.linalg.norm(x) < 1e-9
    # staggered CG on (DD^+)_ee and multi-shift CG
    chi = oracle.gauss(V, 3, 4, 5)
    chi[oracle.parity_mask(L) == 1] = 0
    ks = oracle.Operator("KS_DDDAG_EE", L, U, 0.02)
    y, i3 = oracle.cg(ks, chi, tol=1e-11)
    assert i3["true_rel_residual"] < 1e-10
    shifts = np.logspace(-4, 1, 12)
    ys, i4 = oracle.cgm(ks, chi, shifts, tol=1e-11)
    assert i4["true_rel_residual"] < 1e-10
    for k, s in enumerate(shifts):
        assert ks.true_residual(chi, ys[k], complex(s)) < 1e-10
    # FOM multi-shift with the reference test's complex shifts (TestMultiShiftSolver.cpp:12-111)
    cs = [2, 1, 0.5, 1j, 0.5 + 0.5j, 1 - 1j]
    xs, i5 = oracle.fom_ms(op, b, cs, maxdim=12, restart=200, accuracy=1e-13)
    for k, s in enumerate(cs):
        assert op.true_residual(b, xs[k], complex(s)) < 1e-10
    # BiCGStab-M (CMultiShiftBiCGStab.cpp:73-437) on the same shifts: every shift
    # solved, and the same solutions as the FOM over one Krylov space
    ys, i6 = oracle.bicgstab_ms(op, b, cs, dev_step=10, max_step=100, accuracy=1e-12)
    assert i6["converged"]
    for k, s in enumerate(cs):
        assert op.true_residual(b, ys[k], complex(s)) < 1e-10
        assert np.linalg.norm(ys[k] - xs[k]) < 1e-9 * np.linalg.norm(xs[k])
    # GMRES-M (CMultiShiftGMRES.cpp:113-330): the seed's restarted GMRES, residuals kept collinear
    zs, i7 = oracle.gmres_ms(op, b, cs, maxdim=10, restart=200, accuracy=1e-13, absolute=True)
    assert i7["converged"]
    for k, s in enumerate(cs):
        assert op.true_residual(b, zs[k], complex(s)) < 1e-10
        assert np.linalg.norm(zs[k] - xs[k]) < 1e-9 * np.linalg.norm(xs[k])


def test_wilson_force_is_the_action_derivative(oracle):
    """The Wilson fermion force as the oracle restates _kernelDWilsonForceSU3
    (CFieldFermionWilsonSquareSU3.cu:170-231) is the derivative of the action
    S = phi^+ (DD^+)^-1 phi that CalculateForceS (:1016-1100) differentiates:
    with X = (DD^+)^-1 phi, Y = D^+ X and U_mu(x) -> exp(i e T) U_mu(x) for a
    traceless hermitian T,  dS/de = 2 i Tr(T F_mu(x)).  Checked against central
    finite differences of S (FP64 oracle CG) on random links and generators,
    including links that cross the antiperiodic t boundary."""
    L = (4, 4, 4, 4)
    V = oracle.volume(L)
    kappa = 0.12
    U = oracle.gauge_expH(L, 0xC1A60021, 0.3)
    phi = oracle.gauss(V, 12, 7, 2).reshape(V, 4, 3)

    def action(Ul):
        op = oracle.Operator("WILSON_DDDAG", L, Ul, kappa)
        X, info = oracle.cg(op, phi, tol=1e-13, maxiter=20000)
        assert info["true_rel_residual"] < 1e-12
        return np.vdot(phi, X).real, X

    _, X = action(U)
    Y = oracle.wilson_D(L, U, X, kappa, dagger=True)
    F = oracle.wilson_force(L, U, X, Y, kappa)
    # anti-hermitian and traceless, as Ta makes it
    assert np.abs(F + np.conj(np.transpose(F, (0, 2, 1)))).max() < 1e-14
    assert np.abs(np.trace(F, axis1=1, axis2=2)).max() < 1e-14
    rng = np.random.default_rng(5)
    t_edge = int(np.flatnonzero(np.arange(V) % L[3] == L[3] - 1)[3]) * 4 + 3  # a t link across the boundary
    for link in [t_edge] + [int(v) for v in rng.integers(0, 4 * V, 3)]:
        A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        T = (A + A.conj().T) / 2
        T -= np.trace(T) / 3 * np.eye(3)
        w, Q = np.linalg.eigh(T)
        eps = 1e-5

        def S_at(e):
            U2 = U.copy()
            U2[link] = (Q @ np.diag(np.exp(1j * e * w)) @ Q.conj().T) @ U[link]
            return action(U2)[0]

        dS = (S_at(eps) - S_at(-eps)) / (2 * eps)
        want = (2j * np.trace(T @ F[link])).real
        assert abs(dS - want) <= 1e-6 * max(1.0, abs(want)), (link, dS, want)


def test_ks_force_is_the_rational_action_derivative(oracle):
    """The staggered rational force as the oracle restates _kernelDFermionKSForce
    (Staggered/CFieldFermionKSSU3.cu:216-262) is the derivative of
    S = sum_i a_i phi^+ (DD^+ + b_i)^-1 phi, the U-dependent part of the RHMC
    action whose force CalculateForceS (:412-500) computes from the multi-shift
    solutions phi_i and phi_id = D0 phi_i: dS/de = 2 i Tr(T F_mu(x)) for
    U_mu(x) -> exp(i e T) U_mu(x), on links of every direction, including ones
    that cross the antiperiodic t boundary and the periodic x boundary."""
    L = (4, 4, 4, 4)
    V = oracle.volume(L)
    m = 0.3
    U = oracle.gauge_expH(L, 0xC1A60022, 0.3)
    phi = oracle.gauss(V, 3, 8, 2).reshape(V, 3)
    a = np.array([0.3, 0.7, 1.1])
    b = np.array([0.05, 0.4, 2.0])

    def action(Ul):
        op = oracle.Operator("KS_DDDAG", L, Ul, m)
        xs, info = oracle.cgm(op, phi, list(b), tol=1e-13)
        return sum(a[i] * np.vdot(phi, xs[i]).real for i in range(len(a))), xs

    _, xs = action(U)
    F = oracle.ks_force(L, U, xs, [oracle.ks_D(L, U, x, 0.0) for x in xs], a)
    assert np.abs(F + np.conj(np.transpose(F, (0, 2, 1)))).max() < 1e-14
    assert np.abs(np.trace(F, axis1=1, axis2=2)).max() < 1e-14
    rng = np.random.default_rng(6)
    for link in [4 * (V - 1) + 0, 4 * 63 + 3, 77, 130, 4 * 5 + 0]:
        A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        T = (A + A.conj().T) / 2
        T -= np.trace(T) / 3 * np.eye(3)
        w, Q = np.linalg.eigh(T)
        eps = 1e-5

        def S_at(e):
            U2 = U.copy()
            U2[link] = (Q @ np.diag(np.exp(1j * e * w)) @ Q.conj().T) @ U[link]
            return action(U2)[0]

        dS = (S_at(eps) - S_at(-eps)) / (2 * eps)
        want = (2j * np.trace(T @ F[link])).real
        assert abs(dS - want) <= 1e-6 * max(1.0, abs(want)), (link, dS, want)


def test_gamma_table(oracle):
    """The chiral gamma set and its products (GammaMatrix.h:405-511): GAMMA1..5
    equal the table parsed from the reference header (golden gamma_chiral.json);
    every product equals the matrix product it is defined as; the Clifford
    algebra holds; the next-symmetric index follows CalculateNextSymmetricIndex."""
    gold = json.load(open(os.path.join(GOLDEN, "gamma_chiral.json")))["rows"]
    G = {name: oracle.gamma_matrix(k) for k, name in enumerate(oracle.GAMMAS)}
    for name in ("GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4", "GAMMA5"):
        m = np.zeros((4, 4), np.complex128)
        for r, (c, b) in enumerate(gold[name]):
            m[r, c] = 1j ** b
        np.testing.assert_array_equal(G[name], m)
    g = [None] + [G["GAMMA%d" % k] for k in range(1, 6)]
    prod = {
        "GAMMA51": g[5] @ g[1], "GAMMA52": g[5] @ g[2], "GAMMA53": g[5] @ g[3], "GAMMA54": g[5] @ g[4],
        "GAMMA15": g[1] @ g[5], "GAMMA25": g[2] @ g[5], "GAMMA35": g[3] @ g[5], "GAMMA45": g[4] @ g[5],
        "SIGMA12": 1j * g[2] @ g[1], "SIGMA23": 1j * g[3] @ g[2], "SIGMA31": 1j * g[1] @ g[3],
        "SIGMA12E": 1j * g[1] @ g[2], "SIGMA23E": 1j * g[2] @ g[3], "SIGMA31E": 1j * g[3] @ g[1],
        "SIGMA41": 1j * g[1] @ g[4], "SIGMA42": 1j * g[2] @ g[4], "SIGMA43": 1j * g[3] @ g[4],
        "CHARGECONJG": g[4] @ g[2], "UNITY": np.eye(4),
    }
    for name, m in prod.items():
        np.testing.assert_allclose(G[name], m, atol=1e-15, err_msg=name)
    for mu in range(1, 6):
        for nu in range(1, 6):
            ac = g[mu] @ g[nu] + g[nu] @ g[mu]
            np.testing.assert_allclose(ac, 2 * np.eye(4) * (mu == nu), atol=1e-15)
    for k in range(len(oracle.GAMMAS)):
        idx, z, ns = oracle.gamma(k)
        assert ns == {0: 0, 1: 2, 2: 3, 3: 1}[idx[0]]


def test_meson_and_condensate_contractions(oracle):
    """The oracle's meson contraction and condensate traces equal an independent
    numpy restatement of _kernelCalculateCorrelatorSU3 (CMeasureMesonCorrelator.cu:26-174,
    366-380) and _kernelDotMeasureAll (CMeasureChiralCondensate.cu:38-100) on random fields."""
    L = (4, 4, 2, 6)
    V = oracle.volume(L)
    rng = np.random.default_rng(3)
    props = [rng.normal(size=(V, 4, 3)) + 1j * rng.normal(size=(V, 4, 3)) for _ in range(12)]
    S = np.stack(props)  # [j*3 + a][site][i][b]
    for k in range(len(oracle.GAMMAS)):
        idx, z, ns = oracle.gamma(k)

        def term(i, j, pi, pj):
            return np.sum((np.conj(S[3 * j:3 * j + 3, :, i, :]) * S[3 * pj:3 * pj + 3, :, pi, :]).real, axis=(0, 2))

        res = np.zeros(V)
        for i in range(1, 4):
            for j in range(i + 1, 4):
                zz = z[i] + (((z[j] & 1) << 1) + z[j])
                res += (1.0 - (zz & 2)) * term(i, j, idx[i], idx[j])
        if ns == 0:
            res += 0.5 * sum(term(i, i, i, i) for i in range(4))
        else:
            res += term(0, 0, idx[0], idx[0]) + term(ns, ns, idx[ns], idx[ns])
        want = res.reshape(-1, L[3]).sum(axis=0) * 2 / np.sqrt(V)
        np.testing.assert_allclose(oracle.meson_correlator(L, props, k), want, rtol=1e-12, atol=1e-12)
    eta, psi = props[0], props[1]
    for kind, name in enumerate(["UNITY", "GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4", "GAMMA5", "GAMMA45", "GAMMA1",
                                 "GAMMA2"]):
        G = oracle.gamma_matrix(oracle.GAMMAS.index(name))
        want = np.vdot(eta, np.einsum("rs,xsc->xrc", G, psi)) / V
        assert abs(oracle.condensate(eta, psi, kind) - want) < 1e-12 * abs(want) + 1e-14
