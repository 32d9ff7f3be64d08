"""Parity with the reference itself: the outputs of CLGLib's own CUDA build
(FP64, sm_100a, run on a B200 by tests/golden/make_ref_golden.py) against

* the CPU oracle (this file's CPU tests): D, D^+, DD, DD^+ to 1e-12; the
  oracle's restatements of CSLASolverGMRES, CSLASolverBiCGStab and
  CMultiShiftFOM, run with the reference's parameters, to the reference's
  solutions (1e-9 relative, both solved to a 1e-12 estimate);
* the product's CUDA path (the gpu tests): D, D^+, DD^+ to 1e-12 and the
  solutions of the product's own solvers to 1e-8 relative (the reference's
  solutions are accurate to about 1e-11, the product's to its 1e-10 stop).

A fixture holds, per output y: eight projections <r_k, y> onto fixed probe
fields, y at 67 sampled sites and |y|^2 (see make_ref_golden.py).  The inputs
are regenerated bit for bit from the recorded seeds by the oracle's generator
and checked against the recorded SHA-256 of the bytes the reference was given.
"""
import glob
import hashlib
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_ref_golden as M  # noqa: E402

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))
KAPPA = M.KAPPA
MASS = M.MASS_2AM


def load(name):
    path = os.path.join(GOLDEN, "ref_%s.npz" % name)
    return dict(np.load(path, allow_pickle=False))


def inputs(oracle, fx):
    L = tuple(int(v) for v in fx["dims"])
    V = oracle.volume(L)
    seed = int(fx["seed"])
    if str(fx["links"]) == "haar":
        U = oracle.gauge_haar(L, seed, 1)
    else:
        U = oracle.gauge_expH(L, seed, 0.25)
    ncomp = 12 if str(fx["fermion"]) == "wilson" else 3
    b = oracle.gauss(V, ncomp, seed, 2)
    assert hashlib.sha256(U.tobytes() + b.tobytes()).hexdigest() == str(fx["input_sha256"])
    return L, V, U, b, ncomp


def err(y, fx, key):
    """max over the checks of the relative deviation of y from the reference output `key`."""
    V = y.shape[0]
    flat = y.reshape(V, -1)
    ncomp = flat.shape[1]
    pr = M.probes(V, ncomp)
    ynorm = np.sqrt(float(np.vdot(flat, flat).real))
    proj = np.array([np.vdot(p, flat.reshape(-1)) for p in pr])
    e_proj = max(abs(proj[k] - fx[key + ".proj"][k]) / (np.linalg.norm(pr[k]) * ynorm) for k in range(len(pr)))
    ref_vals = fx[key + ".vals"]
    e_vals = np.abs(flat[fx[key + ".sites"]] - ref_vals).max() / np.abs(ref_vals).max()
    e_norm = abs(ynorm ** 2 - float(fx[key + ".norm2"])) / float(fx[key + ".norm2"])
    return max(e_proj, e_vals, e_norm)


def test_fixtures_present():
    names = {os.path.basename(f) for f in FIXTURES}
    assert {"ref_wilson_haar_8x8x8x8.npz", "ref_wilson_expH_8x8x8x16.npz", "ref_ks_expH_8x8x8x16.npz"} <= names


# ------------------------------------------------------------------ CPU: the oracle against the reference
@pytest.mark.parametrize("name", ["wilson_haar_8x8x8x8", "wilson_expH_8x8x8x16"])
def test_oracle_wilson_operators(oracle, name):
    fx = load(name)
    L, V, U, b, _ = inputs(oracle, fx)
    psi = b.reshape(V, 4, 3)
    D = lambda v, dag=False: oracle.wilson_D(L, U, v, KAPPA, dagger=dag)  # noqa: E731
    assert err(D(psi), fx, "D") < 1e-12
    assert err(D(psi, True), fx, "Ddagger") < 1e-12
    if "DD.proj" in fx:
        assert err(D(D(psi)), fx, "DD") < 1e-12
        assert err(D(D(psi, True)), fx, "DDdagger") < 1e-12


def test_oracle_staggered_operators(oracle):
    fx = load("ks_expH_8x8x8x16")
    L, V, U, b, _ = inputs(oracle, fx)
    D = lambda v, dag=False: oracle.ks_D(L, U, v, MASS, dagger=dag)  # noqa: E731
    assert err(D(b), fx, "D") < 1e-12
    assert err(D(b, True), fx, "Ddagger") < 1e-12
    assert err(D(D(b, True)), fx, "DDdagger") < 1e-12


@pytest.mark.parametrize("name,key,opname", [("wilson_haar_8x8x8x8", "InverseD", "WILSON_D"),
                                             ("wilson_haar_8x8x8x8", "InverseDdagger", "WILSON_DDAG"),
                                             ("wilson_expH_8x8x8x16", "InverseD", "WILSON_D")])
def test_oracle_gmres_matches_reference(oracle, name, key, opname):
    """CSLASolverGMRES (CSolverGMRES.cpp:111-358) restated, GMRES(12), stop on
    |g|^2 < (1e-12 |b|)^2 within the fixture's restart budget.  On the Haar field
    both converge; on the near-critical exp(i 0.25 H) field the reference's
    restarted GMRES stagnates, and the restatement reproduces the stagnated
    iterate (the same true residual, the same x)."""
    fx = load(name)
    L, V, U, b, _ = inputs(oracle, fx)
    restart = int(fx.get(key + ".restart", 2000))
    op = oracle.Operator(opname, L, U, KAPPA)
    bb = b.reshape(V, 4, 3)
    x, info = oracle.gmres(op, bb, maxdim=12, restart=restart, accuracy=(1e-12 * np.linalg.norm(b)) ** 2,
                           absolute=True)
    assert bool(info["converged"]) == bool(int(fx[key + ".ok"]))
    if info["converged"]:
        assert float(fx[key + ".true_res"]) < 1e-10
        assert err(x, fx, key) < 1e-9
    else:
        assert abs(info["true_rel_residual"] - float(fx[key + ".true_res"])) <= 1e-9 * float(fx[key + ".true_res"])
        assert err(x, fx, key) < 1e-9


def test_oracle_bicgstab_matches_reference(oracle):
    """CSLASolverBiCGStab (CSolverBiCGstab.cpp:403-607) with the reference's own omega = <s,t>/|t|^2,
    its default SmallRho 1e-8 (a restart from the current x whenever |rho|^2 falls below it,
    CSolverBiCGstab.cpp:17-24, 481-491) and its stop without the last alpha p update, on the
    config-1 field."""
    fx = load("wilson_haar_8x8x8x8")
    L, V, U, b, _ = inputs(oracle, fx)
    key = "InverseD_bicgstab"
    op = oracle.Operator("WILSON_D", L, U, KAPPA)
    x, info = oracle.bicgstab(op, b.reshape(V, 4, 3), dev_step=1, max_step=500, restart=5,
                              accuracy=(1e-12 * np.linalg.norm(b)) ** 2, absolute=True, small_rho=1e-8,
                              std_omega=False)
    assert int(fx[key + ".ok"]) == int(info["converged"])
    assert err(x, fx, key) < 1e-9


@pytest.mark.parametrize("name,key,opname", [("wilson_haar_8x8x8x8", "MultiShiftD", "WILSON_D"),
                                             ("ks_expH_8x8x8x16", "MultiShiftDDdagger", "KS_DDDAG")])
def test_oracle_fom_ms_matches_reference(oracle, name, key, opname):
    """CMultiShiftFOM (CMultiShiftFOM.cpp:97-270): FOM(30) over one Krylov space, all shifts."""
    fx = load(name)
    L, V, U, b, ncomp = inputs(oracle, fx)
    shifts = fx[key + ".shifts"]
    param = KAPPA if opname.startswith("WILSON") else MASS
    op = oracle.Operator(opname, L, U, param)
    bb = b.reshape((V, 4, 3) if ncomp == 12 else (V, 3))
    xs, info = oracle.fom_ms(op, bb, list(shifts), maxdim=30, restart=2000, accuracy=1e-12 * np.linalg.norm(b),
                             absolute=True)
    for k, c in enumerate(shifts):
        assert float(fx["%s.%d.true_res" % (key, k)]) < 1e-10
        assert err(xs[k], fx, "%s.%d" % (key, k)) < 1e-9, (k, c)


@pytest.mark.parametrize("key,method", [("MultiShiftD_gmres", "gmres"), ("MultiShiftD_bicgstab", "bicgstab")])
def test_oracle_gmres_bicgstab_ms_match_reference(oracle, key, method):
    """CMultiShiftGMRES (CMultiShiftGMRES.cpp:113-330, MaxDim 10, stop on max |beta0_n| < 1e-12) and
    CMultiShiftBiCGStab (CMultiShiftBiCGStab.cpp:73-437, DiviationStep 10, stop on |s|, |s_n| < 1e-12 |b|)
    on the config-1 field with the reference test's shifts."""
    fx = load("wilson_haar_8x8x8x8")
    if key + ".shifts" not in fx:
        pytest.skip("fixture without this solver's outputs")
    L, V, U, b, _ = inputs(oracle, fx)
    shifts = list(fx[key + ".shifts"])
    op = oracle.Operator("WILSON_D", L, U, KAPPA)
    bb = b.reshape(V, 4, 3)
    if method == "gmres":
        xs, info = oracle.gmres_ms(op, bb, shifts, maxdim=10, restart=2000, accuracy=1e-12, absolute=True)
    else:
        xs, info = oracle.bicgstab_ms(op, bb, shifts, dev_step=10, max_step=500, accuracy=1e-12 * np.linalg.norm(b),
                                      absolute=True)
    assert info["converged"] and int(fx[key + ".ok"]) == 1
    for k in range(len(shifts)):
        assert float(fx["%s.%d.true_res" % (key, k)]) < 1e-10
        assert err(xs[k], fx, "%s.%d" % (key, k)) < 1e-9, k


# ------------------------------------------------------------------ GPU: the product against the reference
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wilson_haar_8x8x8x8", "wilson_expH_8x8x8x16"])
def test_product_wilson_vs_reference(ctx, clg, oracle, name):
    fx = load(name)
    L, V, U, b, _ = inputs(oracle, fx)
    lat = clg.Lattice(ctx, L)
    G = clg.CFieldGaugeSU3(lat)
    G.InitialWithByte(U)
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    for op, key in [(clg.EFO_F_D, "D"), (clg.EFO_F_Ddagger, "Ddagger"), (clg.EFO_F_DDdagger, "DDdagger")]:
        if key + ".proj" not in fx:
            continue
        f.from_numpy(b.reshape(V, 4, 3))
        f.ApplyOperator(op, G)
        assert err(f.to_numpy(), fx, key) < 1e-12, key
    # the product's solvers (FP16 / FP32 inner, FP64 true residual 1e-10) against
    # the reference's solutions where the reference converged; where its GMRES(12)
    # stagnated (the exp(i 0.25 H) field) the product still reaches 1e-10
    src = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    src.from_numpy(b.reshape(V, 4, 3))
    for key, op, name in [("InverseD", clg.EFO_F_D, "WILSON_D"), ("InverseDdagger", clg.EFO_F_Ddagger, "WILSON_DDAG")]:
        if key + ".proj" not in fx:
            continue
        o = oracle.Operator(name, L, U, KAPPA)
        for S in (clg.CSLASolverCG(ctx, inner_precision=clg.HALF, tol_true_rel=1e-10),
                  clg.CSLASolverGMRES(ctx, inner_precision=clg.SINGLE, tol_true_rel=1e-10, MaxDim=12)):
            x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
            info = S.Solve(x, src, G, op, raise_on_fail=False)[0]
            if int(fx[key + ".ok"]):
                assert err(x.to_numpy(), fx, key) < 1e-8, key
            elif S.KIND == clg.SOLVER_CG:  # restarted GMRES stagnates here for the product as well
                assert info["status"] == 0 and o.true_residual(b.reshape(V, 4, 3), x.to_numpy()) <= 1e-10


@pytest.mark.gpu
def test_product_staggered_vs_reference(ctx, clg, oracle):
    fx = load("ks_expH_8x8x8x16")
    L, V, U, b, _ = inputs(oracle, fx)
    lat = clg.Lattice(ctx, L)
    G = clg.CFieldGaugeSU3(lat)
    G.InitialWithByte(U)
    f = clg.CFieldFermionKSSU3(lat, MASS)
    for op, key in [(clg.EFO_F_D, "D"), (clg.EFO_F_Ddagger, "Ddagger"), (clg.EFO_F_DDdagger, "DDdagger")]:
        f.from_numpy(b)
        f.ApplyOperator(op, G)
        assert err(f.to_numpy(), fx, key) < 1e-12, key
    # the product's multi-shift solve of (DD^+ + sigma) on the full lattice against CMultiShiftFOM's
    key = "MultiShiftDDdagger"
    shifts = [complex(c) for c in fx[key + ".shifts"]]
    src = clg.CFieldFermionKSSU3(lat, MASS)
    src.from_numpy(b)
    xs = [clg.CFieldFermionKSSU3(lat, MASS) for _ in shifts]
    S = clg.CMultiShiftCG(ctx, inner_precision=clg.SINGLE)
    S.Solve(xs, [c.real for c in shifts], src, G, clg.EFO_F_DDdagger)
    for k in range(len(shifts)):
        assert err(xs[k].to_numpy(), fx, "%s.%d" % (key, k)) < 1e-8, k


@pytest.mark.gpu
def test_product_multishift_wilson_vs_reference(ctx, clg, oracle):
    """(D + c) x = b for the reference test's complex shifts against CMultiShiftFOM's solutions."""
    fx = load("wilson_haar_8x8x8x8")
    L, V, U, b, _ = inputs(oracle, fx)
    lat = clg.Lattice(ctx, L)
    G = clg.CFieldGaugeSU3(lat)
    G.InitialWithByte(U)
    key = "MultiShiftD"
    shifts = [complex(c) for c in fx[key + ".shifts"]]
    src = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA)
    src.from_numpy(b.reshape(V, 4, 3))
    xs = [clg.CFieldFermionWilsonSquareSU3(lat, KAPPA) for _ in shifts]
    S = clg.CMultiShiftFOM(ctx, inner_precision=clg.SINGLE)
    S.Solve(xs, shifts, src, G, clg.EFO_F_D)
    for k in range(len(shifts)):
        assert err(xs[k].to_numpy(), fx, "%s.%d" % (key, k)) < 1e-8, k
