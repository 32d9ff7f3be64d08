"""Gauge-configuration and fermion-field files (CFieldGaugeSU3::InitialFieldWithFile,
CField::SaveToFile, SaveToCompressedFile; TestConfigurationFileIO.cpp) through
the library, pinned to the reference's own Bridge++ configuration and the MD5
of its binary file (tests/golden/fileio.json)."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def bridgepp(clg, ctx):
    g = np.load(os.path.join(GOLDEN, "bridgepp_4x4x4x8.npz"))
    lat = clg.Lattice(ctx, tuple(int(d) for d in g["dims"]))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialWithByte(g["links"], layout=clg.LAYOUT_BRIDGEPP)
    return lat, U, g


def test_bridgepp_binary_matches_the_reference_file(ctx, clg, tmp_path):
    """The reference's 4^3x8 configuration written as a Bridge++ binary file has
    the MD5 of the reference's own bridgepp_conf_binary.dat; read back, text and
    binary give the known plaquette 0.625129946974942 (TestConfigurationFileIO.cpp:12-38)."""
    want = json.load(open(os.path.join(GOLDEN, "fileio.json")))["bridgepp_conf_binary.dat"]
    lat, U, g = bridgepp(clg, ctx)
    p = str(tmp_path / "conf.bin")
    assert U.SaveToFile(p, clg.FILE_BRIDGEPP_BIN) == want["md5"]
    assert os.path.getsize(p) == want["bytes"]
    assert hashlib.md5(open(p, "rb").read()).hexdigest() == want["md5"]
    for fmt, path in ((clg.FILE_BRIDGEPP_BIN, p), (clg.FILE_BRIDGEPP_TXT, str(tmp_path / "conf.txt"))):
        if fmt == clg.FILE_BRIDGEPP_TXT:
            U.SaveToFile(path, fmt)
        V = clg.CFieldGaugeSU3(lat)
        V.InitialFieldWithFile(path, fmt)
        assert abs(V.plaquette() - float(g["plaquette"])) < 1e-12
        assert np.array_equal(V.CopyDataOut(), U.CopyDataOut())


def test_clgbin_double_and_float(ctx, clg, tmp_path):
    """CLGBin double is the CLGBin-ordered doubles of the links (MD5 of exactly
    those bytes) and reads back bit for bit; CLGBin float to float rounding."""
    lat = clg.Lattice(ctx, (4, 6, 4, 8))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 0xC1A60071, 1)
    Uh = U.CopyDataOut()
    p = str(tmp_path / "u.con")
    assert U.SaveToFile(p, clg.FILE_CLGBIN_DOUBLE) == hashlib.md5(Uh.tobytes()).hexdigest()
    V = clg.CFieldGaugeSU3(lat)
    V.InitialFieldWithFile(p, clg.FILE_CLGBIN_DOUBLE)
    assert np.array_equal(V.CopyDataOut(), Uh)
    pf = str(tmp_path / "u.conf")
    md5f = U.SaveToFile(pf, clg.FILE_CLGBIN_FLOAT)
    assert md5f == hashlib.md5(Uh.view(np.float64).astype(np.float32).tobytes()).hexdigest()
    V.InitialFieldWithFile(pf, clg.FILE_CLGBIN_FLOAT)
    assert np.abs(V.CopyDataOut() - Uh).max() < 1e-7
    # the known-answer shape of TestFileDOUBLE / TestFileFloat: sum |U|^2 = 3 per link
    assert abs(np.vdot(Uh, Uh).real - 3 * 4 * lat.volume) < 1e-9


@pytest.mark.parametrize("kind", ["haar", "expH", "identity"])
def test_compressed_round_trip(ctx, clg, tmp_path, kind):
    """SaveToCompressedFile stores A = log U (anti-hermitian: A01, A02, A12,
    imaginary diagonal); InitialWithByteCompressed rebuilds U = exp A.  FP64
    files reproduce the links to 1e-13 (the reference test allows 1e-8 on
    sum |dU|^2), float files to float rounding."""
    from scipy.linalg import expm

    lat = clg.Lattice(ctx, (4, 4, 4, 8))
    U = clg.CFieldGaugeSU3(lat)
    if kind == "haar":
        U.InitialField(clg.GAUGE_HAAR, 0xC1A60072, 1)
    elif kind == "expH":
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60073, 1, 0.3)
    else:
        U.InitialField(clg.GAUGE_IDENTITY)
    Uh = U.CopyDataOut()
    p = str(tmp_path / "c.con")
    U.SaveToFile(p, clg.FILE_CLGBIN_COMPRESSED)
    raw = np.fromfile(p, dtype=np.float64).reshape(-1, 9)
    assert raw.shape[0] == 4 * lat.volume
    # the stored numbers are the logarithm: exp of the rebuilt A is U
    for l in [0, 7, 1000, 4 * lat.volume - 1]:
        o = raw[l]
        A = np.array([[1j * o[6], o[0] + 1j * o[1], o[2] + 1j * o[3]],
                      [-o[0] + 1j * o[1], 1j * o[7], o[4] + 1j * o[5]],
                      [-o[2] + 1j * o[3], -o[4] + 1j * o[5], 1j * o[8]]])
        assert np.abs(expm(A) - Uh[l]).max() < 1e-13
        assert np.abs(np.linalg.eigvals(A).imag).max() <= np.pi + 1e-12  # principal branch
    V = clg.CFieldGaugeSU3(lat)
    V.InitialFieldWithFile(p, clg.FILE_CLGBIN_COMPRESSED)
    assert np.abs(V.CopyDataOut() - Uh).max() < 1e-13
    pf = str(tmp_path / "c.conf")
    U.SaveToFile(pf, clg.FILE_CLGBIN_COMPRESSED_FLOAT)
    assert os.path.getsize(pf) == 4 * lat.volume * 9 * 4
    V.InitialFieldWithFile(pf, clg.FILE_CLGBIN_COMPRESSED_FLOAT)
    assert np.abs(V.CopyDataOut() - Uh).max() < 5e-6


def test_fermion_files(ctx, clg, tmp_path):
    """TestFileIOCLG: a fermion field saved and read back is the same field."""
    lat = clg.Lattice(ctx, (4, 4, 4, 8))
    for cls, nc in ((clg.CFieldFermionWilsonSquareSU3, 12), (clg.CFieldFermionKSSU3, 3)):
        f = cls(lat, 0.1, nrhs=2)
        f.InitialField(clg.SOURCE_GAUSS, 0xC1A60074, 2, rhs=1)
        h = f.to_numpy(1)
        p = str(tmp_path / "f.con")
        assert f.SaveToFile(p, clg.FILE_CLGBIN_DOUBLE, rhs=1) == hashlib.md5(h.tobytes()).hexdigest()
        g = cls(lat, 0.1)
        g.InitialFieldWithFile(p, clg.FILE_CLGBIN_DOUBLE)
        assert np.array_equal(g.to_numpy(), h)
        f.SaveToFile(p, clg.FILE_CLGBIN_FLOAT, rhs=1)
        g.InitialFieldWithFile(p, clg.FILE_CLGBIN_FLOAT)
        assert np.abs(g.to_numpy() - h).max() < 1e-6 * np.abs(h).max()


def test_file_errors(ctx, clg, tmp_path):
    """Wrong sizes, missing files, unknown formats and non-SU(3) compressed saves are errors."""
    lat = clg.Lattice(ctx, (4, 4, 4, 4))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 3, 1)
    p = str(tmp_path / "u.con")
    U.SaveToFile(p)
    big = clg.Lattice(ctx, (4, 4, 4, 8))
    V = clg.CFieldGaugeSU3(big)
    with pytest.raises(clg.CLGError):
        V.InitialFieldWithFile(p, clg.FILE_CLGBIN_DOUBLE)
    with pytest.raises(clg.CLGError):
        V.InitialFieldWithFile(str(tmp_path / "missing.con"))
    with pytest.raises(clg.CLGError):
        U.SaveToFile(p, 17)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_ZERO)
    with pytest.raises(clg.CLGError):
        F.SaveToFile(str(tmp_path / "z.con"), clg.FILE_CLGBIN_COMPRESSED)
    f = clg.CFieldFermionWilsonSquareSU3(lat, 0.1)
    with pytest.raises(clg.CLGError):
        f.SaveToFile(p, clg.FILE_BRIDGEPP_BIN)
