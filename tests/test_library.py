"""CPU-side checks of the C ABI library: it builds, loads, and exports every
entry point declared in include/clg_b200.h (no device computation)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "clg_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(clg_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib_path():
    from cudalatticegauge_b200 import build

    return build.build()


def test_exports_every_header_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (clg_[a-z0-9_]+)$", out, flags=re.M))
    missing = [f for f in header_functions() if f not in exported]
    assert not missing, missing
    assert len(header_functions()) >= 30


def test_library_loads_and_binds_every_symbol(lib_path):
    import cudalatticegauge_b200 as clg

    lib = clg.load_library(lib_path)
    names = {n for n, _, _ in clg.SIGNATURES}
    assert names == set(header_functions())
    assert lib.clg_status_string(clg.ERR_NOT_CONVERGED) == b"solver did not converge"


def test_built_for_sm100a(lib_path):
    """Every nvcc command of the build targets sm_100a and nothing else (read
    from the build recipe; no binary tool looks into the library)."""
    from cudalatticegauge_b200 import build

    flags = list(build.NVCC_FLAGS)
    i = flags.index("-gencode")
    assert flags[i + 1] == "arch=compute_100a,code=sm_100a"
    assert flags.count("-gencode") == 1
    assert not any(f.startswith("-arch") for f in flags)


def test_no_device_is_an_error_not_a_crash(lib_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import cudalatticegauge_b200 as clg

    with pytest.raises(clg.CLGError) as e:
        clg.Context(0)
    assert e.value.status == clg.ERR_NO_DEVICE


def test_md5_rfc1321_vectors(lib_path):
    """CLGMD5Hash: the RFC 1321 test suite, and hashlib on lengths around the
    64-byte block and padding boundaries (host code, no GPU)."""
    import hashlib

    import cudalatticegauge_b200 as clg

    clg.load_library(lib_path)
    suite = {
        b"": "d41d8cd98f00b204e9800998ecf8427e",
        b"a": "0cc175b9c0f1b6a831c399e269772661",
        b"abc": "900150983cd24fb0d6963f7d28e17f72",
        b"message digest": "f96b697d7cb7938d525a2f31aaf161d0",
        b"abcdefghijklmnopqrstuvwxyz": "c3fcd3d76192e4007dfb496cca67e13b",
        b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789": "d174ab98d277d9f5a5611c2c9f419d9f",
        b"1234567890" * 8: "57edf4a22be3c955ac49da2e2107b67a",
    }
    for msg, want in suite.items():
        assert clg.md5(msg) == want
    rng = np.random.default_rng(11)
    for n in (55, 56, 57, 63, 64, 65, 119, 120, 128, 1 << 20):
        b = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert clg.md5(b) == hashlib.md5(b).hexdigest(), n


def test_small_dense_eigensolver(lib_path):
    """The host eigensolver of the recycled solver: A x = w x and A x = w B x
    (B Hermitian positive definite) on random complex matrices up to order 33,
    against numpy's eigenvalues; residuals at rounding level; a Hermitian
    matrix with repeated eigenvalues."""
    import cudalatticegauge_b200 as clg

    clg.load_library(lib_path)
    rng = np.random.default_rng(7)
    for n in (1, 2, 3, 5, 10, 20, 33):
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        w, X = clg.small_eig(A)
        assert np.abs(A @ X - X * w).max() < 1e-12 * np.abs(A).max()
        np.testing.assert_allclose(np.sort(np.abs(w)), np.sort(np.abs(np.linalg.eigvals(A))), rtol=1e-10)
        M = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        B = M @ M.conj().T + n * np.eye(n)
        w2, X2 = clg.small_eig(A, B)
        assert np.abs(A @ X2 - (B @ X2) * w2).max() < 1e-12 * np.abs(A).max() * np.abs(B).max()
    Q, _ = np.linalg.qr(rng.normal(size=(12, 12)) + 1j * rng.normal(size=(12, 12)))
    H = Q @ np.diag([1, 1, 1, 2, 2, 3, 4, 5, 6, 7, 8, 9.0]) @ Q.conj().T
    w, X = clg.small_eig(H)
    assert np.abs(H @ X - X * w).max() < 1e-12
    np.testing.assert_allclose(np.sort(w.real), [1, 1, 1, 2, 2, 3, 4, 5, 6, 7, 8, 9], atol=1e-12)
