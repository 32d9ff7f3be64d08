"""Every launch variant of the Wilson hop against the FP64 oracle.

The autotuner picks one variant per operator and lattice, so the tuned runs
of the other tests exercise only the winner.  Here each variant is pinned
through CLG_HOP_CONFIG ("<variant>:<block>", read when a context is created):
0 = plain, 1 = capped at 80 registers, 2 = capped at 72.  Lattices with a partial last
block per checkerboard and two right-hand sides (the rhs strides and FP16
norms) are included.  Tolerances as in test_gpu_dslash: FP32 2e-6, FP16 storage 5e-3.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
KAPPA = 0.1355
CONFIGS = ["0:64", "0:128", "0:256", "1:64", "1:128", "1:256", "2:64"]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def pinned(clg, monkeypatch_module):
    made = {}

    def get(cfg):
        if cfg not in made:
            monkeypatch_module.setenv("CLG_HOP_CONFIG", cfg)
            made[cfg] = clg.Context(0)
            monkeypatch_module.delenv("CLG_HOP_CONFIG")
        return made[cfg]

    yield get
    for c in made.values():
        c.close()


@pytest.fixture(scope="module")
def monkeypatch_module():
    mp = pytest.MonkeyPatch()
    yield mp
    mp.undo()


@pytest.mark.parametrize("cfg", CONFIGS)
@pytest.mark.parametrize("prec,tol", [(1, 2e-6), (2, 5e-3)])
@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (4, 6, 4, 10)])
def test_hop_variant(clg, oracle, pinned, cfg, prec, tol, dims):
    ctx = pinned(cfg)
    lat = clg.Lattice(ctx, dims)
    L = lat.dims
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 0xC1A60007, 1)
    Uh = U.CopyDataOut()
    n = 2
    src = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=n)
    for r in range(n):
        src.InitialField(clg.SOURCE_GAUSS, 40 + r, 2, rhs=r)
    psi = [src.to_numpy(r) for r in range(n)]
    for dagger in (False, True):
        f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, precision=prec, nrhs=n)
        for r in range(n):
            f.from_numpy(psi[r], r)
        (f.Ddagger if dagger else f.D)(U)
        for r in range(n):
            want = oracle.wilson_D(L, Uh, psi[r], KAPPA, dagger=dagger)
            assert rel(f.to_numpy(r), want) < tol, (cfg, prec, dims, dagger, r)
        f.close()
    src.close()
