"""Every launch variant of the Wilson hop against the FP64 oracle.

The autotuner picks one variant per operator and lattice, so the tuned runs
of the other tests exercise only the winner.  Here each variant is pinned
through CLG_HOP_CONFIG ("<variant>:<block>", read when a context is created):
0 = plain, 1 = capped at 80 registers, 2 = capped at 72, 3 = FP64 capped at
128; 16..19 the FP64 / FP32 tile form (32 sites per block, links staged once
for all right-hand sides; bit 0 the register cap, bit 1 the blocked order).  Lattices with a partial last
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


@pytest.mark.parametrize("cfg", CONFIGS + ["3:64", "3:128", "3:256", "16:128", "17:96", "18:256", "19:64"])
@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 2e-6), (2, 5e-3)])
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


def _context_with(clg, name, value):
    import os

    old = os.environ.get(name)
    os.environ[name] = value
    try:
        return clg.Context(0)
    finally:
        if old is None:
            del os.environ[name]
        else:
            os.environ[name] = old


@pytest.fixture(scope="module")
def ctx_pair(clg):
    """A context whose FP16 Wilson hops compute pairs of right-hand sides
    (CLG_HOP_PAIR=1)."""
    c = _context_with(clg, "CLG_HOP_PAIR", "1")
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_single(clg):
    """A context whose FP16 Wilson hops keep one right-hand side per thread
    (CLG_HOP_PAIR=0; the default context lets the autotuner time both)."""
    c = _context_with(clg, "CLG_HOP_PAIR", "0")
    yield c
    c.close()


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (6, 10, 14, 12)])
@pytest.mark.parametrize("nrhs", [2, 3, 5])
@pytest.mark.parametrize("op", ["MEE", "MEE_DAG"])
def test_fp16_pair_hop_bit_identical(ctx, ctx_single, ctx_pair, clg, dims, nrhs, op):
    """The paired FP16 hop (two right-hand sides per thread, planar) gives the
    same bits as the one-rhs kernel; odd counts leave one unpaired member.  The
    default context, whose autotuner picks either form, gives them too."""
    outs = []
    for c in (ctx_single, ctx_pair, ctx):
        lat = clg.Lattice(c, dims)
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
        f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF, nrhs=nrhs)
        for r in range(nrhs):
            f.InitialField(clg.SOURCE_GAUSS, 300 + r, 2, rhs=r)
        f.ApplyOperator(getattr(clg, "OP_" + op), U)
        outs.append([f.to_numpy(r) for r in range(nrhs)])
    for r in range(nrhs):
        np.testing.assert_array_equal(outs[0][r], outs[1][r])
        np.testing.assert_array_equal(outs[0][r], outs[2][r])


@pytest.mark.parametrize("nrhs", [2, 3])
def test_fp16_pair_cg_epilogues_identical(ctx, ctx_single, ctx_pair, clg, oracle, nrhs):
    """The fused CGNE iteration with paired hops and epilogues (CgHopAlpha,
    CgHopUpdate over two right-hand sides per block) runs the same iterations
    and gives the same solutions as the one-rhs kernels, and so does the
    default context with the form its autotuner chose."""
    res = []
    for c in (ctx_single, ctx_pair, ctx):
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
        b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
        for r in range(nrhs):
            b.InitialField(clg.SOURCE_GAUSS, 400 + r, 2, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
        S = clg.CSLASolverCG(c, inner_precision=clg.HALF, tol_true_rel=1e-10)
        infos = S.Solve(x, b, U, clg.EFO_F_D)
        res.append(([i["iterations"] for i in infos], [x.to_numpy(r) for r in range(nrhs)], U.CopyDataOut(),
                    [b.to_numpy(r) for r in range(nrhs)]))
    assert res[0][0] == res[1][0] == res[2][0]
    op = oracle.Operator("WILSON_D", (8, 8, 8, 16), res[0][2], KAPPA)
    for r in range(nrhs):
        np.testing.assert_array_equal(res[0][1][r], res[1][1][r])
        np.testing.assert_array_equal(res[0][1][r], res[2][1][r])
        assert op.true_residual(res[0][3][r], res[0][1][r]) <= 1e-10


@pytest.mark.parametrize("cfg", ["0:64", "0:128", "0:256", "1:64", "1:128", "1:256"])
def test_fp16_pair_variants_vs_oracle(clg, oracle, cfg):
    """Each paired launch variant (CLG_HOP_PAIR="<variant>:<block>") against the
    FP64 oracle on a lattice with a partial last block, three right-hand sides."""
    import os

    os.environ["CLG_HOP_PAIR"] = cfg
    try:
        c = clg.Context(0)
    finally:
        del os.environ["CLG_HOP_PAIR"]
    try:
        dims = (6, 10, 14, 12)
        lat = clg.Lattice(c, dims)
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
        Uh = U.CopyDataOut()
        pm = clg.eo_parity(dims)
        f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF, nrhs=3)
        src = []
        for r in range(3):
            g = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN)
            g.InitialField(clg.SOURCE_GAUSS, 500 + r, 2)
            src.append(g.to_numpy())
            f.from_numpy(src[-1], rhs=r)
        f.ApplyOperator(clg.OP_MEE, U)
        for r in range(3):
            want = oracle.wilson_mee(dims, Uh, src[r], KAPPA)[pm == 0]
            assert rel(f.to_numpy(r)[pm == 0], want) < 5e-3
    finally:
        c.close()


TILE_CONFIGS = ["8:0", "8:1", "4:1", "3:1", "4:3", "7:2", "4:4", "4:7", "2:5"]


@pytest.fixture(scope="module")
def ctx_tiles(clg):
    """Contexts whose FP16 Wilson hops over two or more right-hand sides use
    the tile form (CLG_HOP_TILE="<warps>:<variant>": 32 sites per block, the
    links staged once in shared memory for all right-hand sides; variants 0-3:
    bit 0 caps the registers at 80, bit 1 walks the tiles in chunks of y-rows;
    4-7 cap at 72, or at 64 with bit 0)."""
    made = {}

    def get(cfg):
        if cfg not in made:
            made[cfg] = _context_with(clg, "CLG_HOP_TILE", cfg)
        return made[cfg]

    yield get
    for c in made.values():
        c.close()


@pytest.mark.parametrize("cfg", TILE_CONFIGS)
@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (6, 10, 14, 12)])
@pytest.mark.parametrize("nrhs", [2, 5, 9])
@pytest.mark.parametrize("op", ["MEE", "MEE_DAG"])
def test_fp16_tile_hop_bit_identical(ctx_single, ctx_tiles, clg, cfg, dims, nrhs, op):
    """The tile form gives the same bits as the one-rhs kernel, with a partial
    last tile (6x10x14x12: 2520 sites per checkerboard, site order) and more
    right-hand sides than warps; on 8^4 the blocked order covers every tile."""
    outs = []
    for c in (ctx_single, ctx_tiles(cfg)):
        lat = clg.Lattice(c, dims)
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
        f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF, nrhs=nrhs)
        for r in range(nrhs):
            f.InitialField(clg.SOURCE_GAUSS, 600 + r, 2, rhs=r)
        f.ApplyOperator(getattr(clg, "OP_" + op), U)
        outs.append([f.to_numpy(r) for r in range(nrhs)])
    for r in range(nrhs):
        np.testing.assert_array_equal(outs[0][r], outs[1][r])


@pytest.mark.parametrize("cfg", ["8:1", "3:0", "4:3", "4:6", "4:5"])
def test_fp16_tile_cg_epilogues(ctx_single, ctx_tiles, clg, oracle, cfg):
    """The fused CGNE iteration with the tile form's epilogues (CgHopAlpha,
    CgHopUpdate reduced per tile and in two levels) converges like the one-rhs
    kernels, to 1e-10 by the oracle's residual, on five right-hand sides that
    finish at different iterations (the finished ones are skipped)."""
    nrhs = 5
    res = []
    for c in (ctx_single, ctx_tiles(cfg)):
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
        b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
        for r in range(nrhs):
            b.InitialField(clg.SOURCE_GAUSS if r % 2 else clg.SOURCE_Z2, 700 + r, 2, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
        S = clg.CSLASolverCG(c, inner_precision=clg.HALF, tol_true_rel=1e-10)
        infos = S.Solve(x, b, U, clg.EFO_F_D)
        res.append(([i["iterations"] for i in infos], [x.to_numpy(r) for r in range(nrhs)], U.CopyDataOut(),
                    [b.to_numpy(r) for r in range(nrhs)]))
    op = oracle.Operator("WILSON_D", (8, 8, 8, 16), res[1][2], KAPPA)
    for r in range(nrhs):
        assert abs(res[0][0][r] - res[1][0][r]) <= max(3, res[0][0][r] // 20), (res[0][0], res[1][0])
        assert op.true_residual(res[1][3][r], res[1][1][r]) <= 1e-10


MMA_CONFIGS = ["8:8", "8:11"]


@pytest.mark.parametrize("cfg", MMA_CONFIGS)
@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (6, 10, 14, 12)])
@pytest.mark.parametrize("nrhs", [2, 5, 17])
@pytest.mark.parametrize("dagger", [False, True])
def test_fp16_mma_hop_vs_oracle(ctx_tiles, clg, oracle, cfg, dims, nrhs, dagger):
    """The tensor-core form (CLG_HOP_TILE="8:8", "8:11": mma.sync colour
    products, 8 sites per block, right-hand sides in groups of 16) against the
    FP64 oracle's M_ee (and M_ee^+) within the FP16 tolerance, with a partial
    last tile (6x10x14x12) and a partial last group (17 rhs)."""
    c = ctx_tiles(cfg)
    lat = clg.Lattice(c, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
    Uh = U.CopyDataOut()
    pm = clg.eo_parity(dims)
    f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF, nrhs=nrhs)
    src = []
    for r in range(nrhs):
        g = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN)
        g.InitialField(clg.SOURCE_GAUSS, 800 + r, 2)
        src.append(g.to_numpy())
        f.from_numpy(src[-1], rhs=r)
    f.ApplyOperator(clg.OP_MEE_DAG if dagger else clg.OP_MEE, U)
    for r in range(nrhs):
        want = oracle.wilson_mee(dims, Uh, src[r], KAPPA, dagger=dagger)[pm == 0]
        assert rel(f.to_numpy(r)[pm == 0], want) < 5e-3, (cfg, dims, nrhs, dagger, r)


@pytest.mark.parametrize("cfg", MMA_CONFIGS)
def test_fp16_mma_cg_epilogues(ctx_tiles, clg, oracle, cfg):
    """CGNE with the tensor-core form's fused epilogues converges to 1e-10 by
    the oracle's residual on five right-hand sides that finish at different
    iterations."""
    nrhs = 5
    c = ctx_tiles(cfg)
    lat = clg.Lattice(c, (8, 8, 8, 16))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
    for r in range(nrhs):
        b.InitialField(clg.SOURCE_GAUSS if r % 2 else clg.SOURCE_Z2, 700 + r, 2, rhs=r)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=nrhs)
    S = clg.CSLASolverCG(c, inner_precision=clg.HALF, tol_true_rel=1e-10)
    infos = S.Solve(x, b, U, clg.EFO_F_D)
    op = oracle.Operator("WILSON_D", (8, 8, 8, 16), U.CopyDataOut(), KAPPA)
    for r in range(nrhs):
        assert infos[r]["status"] == 0
        assert op.true_residual(b.to_numpy(r), x.to_numpy(r)) <= 1e-10


@pytest.mark.parametrize("cfg", ["16:128", "19:256"])
@pytest.mark.parametrize("prec", [0, 1])
def test_tileN_bit_identical(clg, pinned, cfg, prec):
    """The FP64 tile form gives the same bits as the one-rhs kernel (pinned
    "0:128") on 5 right-hand sides, in D and D^+; FP32 agrees to its rounding
    (the compiler contracts the products of the rebuilt third link row into
    FMAs differently in the two kernels)."""
    outs = []
    for c in (pinned("0:128"), pinned(cfg)):
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
        f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, precision=prec, nrhs=5)
        for r in range(5):
            f.InitialField(clg.SOURCE_GAUSS, 900 + r, 2, rhs=r)
        f.D(U)
        f.Ddagger(U)
        outs.append([f.to_numpy(r) for r in range(5)])
    for r in range(5):
        if prec == 0:
            np.testing.assert_array_equal(outs[0][r], outs[1][r])
        else:
            assert rel(outs[1][r], outs[0][r]) < 2e-6


@pytest.mark.parametrize("cfg", ["17:128", "18:224"])
def test_tileN_cg_fp64(clg, oracle, pinned, cfg):
    """FP64 CGNE with the tile form's fused epilogues (four right-hand sides,
    7 warps for 4 rhs in "18:224") converges to 1e-10 by the oracle."""
    c = pinned(cfg)
    lat = clg.Lattice(c, (8, 8, 8, 16))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
    b = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=4)
    for r in range(4):
        b.InitialField(clg.SOURCE_GAUSS, 950 + r, 2, rhs=r)
    x = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, nrhs=4)
    S = clg.CSLASolverCG(c, inner_precision=clg.DOUBLE, tol_true_rel=1e-10)
    infos = S.Solve(x, b, U, clg.EFO_F_D)
    op = oracle.Operator("WILSON_D", (8, 8, 8, 16), U.CopyDataOut(), KAPPA)
    for r in range(4):
        assert infos[r]["status"] == 0
        assert op.true_residual(b.to_numpy(r), x.to_numpy(r)) <= 1e-10


def test_tune_file_round_trip(clg, tmp_path):
    """CLG_TUNE_FILE: a context writes the autotuner's choices when it is
    destroyed and the next context reads them back (clg_context_tuned shows
    the same forms), so a later run launches the kernels an earlier run chose."""
    import os

    path = str(tmp_path / "tune.txt")
    old = os.environ.get("CLG_TUNE_FILE")
    os.environ["CLG_TUNE_FILE"] = path
    try:
        c = clg.Context(0)
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
        f = clg.CFieldFermionWilsonSquareSU3(lat, KAPPA, subset=clg.EVEN, precision=clg.HALF, nrhs=4)
        for r in range(4):
            f.InitialField(clg.SOURCE_GAUSS, 990 + r, 2, rhs=r)
        f.ApplyOperator(clg.OP_MEE, U)
        first = c.tuned()
        assert any(k.startswith("wilson_p2_") and k.endswith("_auto") for k in first)
        for o in (f, U, lat):
            o.close()
        c.close()
        text = open(path).read()
        assert all(f"{k}=" in text for k in first)
        c2 = clg.Context(0)
        assert c2.tuned() == first
        c2.close()
    finally:
        if old is None:
            del os.environ["CLG_TUNE_FILE"]
        else:
            os.environ["CLG_TUNE_FILE"] = old


@pytest.mark.parametrize("cfg", ["16:128", "19:256"])
@pytest.mark.parametrize("prec", [0, 1])
def test_staggered_tile(clg, oracle, pinned, cfg, prec):
    """The staggered tile form (links staged once per tile for all right-hand
    sides) against the one-rhs kernel (pinned "0:128"): the same bits in FP64,
    FP32 to its rounding; and against the oracle's D on 5 right-hand sides."""
    m = 0.02
    outs = []
    for c in (pinned("0:128"), pinned(cfg)):
        lat = clg.Lattice(c, (8, 8, 8, 16))
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60004, 1, 0.25)
        Uh = U.CopyDataOut()
        f64 = clg.CFieldFermionKSSU3(lat, m)
        f = clg.CFieldFermionKSSU3(lat, m, precision=prec, nrhs=5)
        chis = []
        for r in range(5):
            f64.InitialField(clg.SOURCE_GAUSS, 970 + r, 2)
            chis.append(f64.to_numpy())
            f.from_numpy(chis[-1], r)
        f.D(U)
        outs.append([f.to_numpy(r) for r in range(5)])
    for r in range(5):
        if prec == 0:
            np.testing.assert_array_equal(outs[0][r], outs[1][r])
        else:
            assert rel(outs[1][r], outs[0][r]) < 2e-6
        assert rel(outs[1][r], oracle.ks_D((8, 8, 8, 16), Uh, chis[r], m)) < (1e-12 if prec == 0 else 2e-6)
