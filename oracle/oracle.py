"""ctypes wrapper around the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py`` -- never by the product package.

Arrays are numpy ``complex128`` in the reference's CLGBin order:
gauge ``[V*4, 3, 3]`` (link = site*4 + mu), Wilson spinor ``[V, 4, 3]``,
staggered vector ``[V, 3]``; site = ((x*Ly + y)*Lz + z)*Lt + t.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(_HERE, f) for f in ("clg_oracle.c", "clg_oracle_fields.c", "clg_oracle_measure.c", "clg_oracle.h")]
    if force or not os.path.exists(_LIB_PATH) or any(
        os.path.getmtime(s) > os.path.getmtime(_LIB_PATH) for s in srcs
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Lat(C.Structure):
    _fields_ = [("L", C.c_int * 4), ("bc", C.c_int * 4)]


class Op(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("lat", Lat),
        ("U", C.c_void_p),
        ("param", C.c_double),
        ("tmp", C.c_void_p),
        ("tmp2", C.c_void_p),
    ]


class Info(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("restarts", C.c_int),
        ("converged", C.c_int),
        ("last_deviation", C.c_double),
        ("true_rel_residual", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


OP = dict(
    WILSON_D=0, WILSON_DDAG=1, WILSON_DDDAG=2, WILSON_DD=3, WILSON_MEE=4, WILSON_MEE_DAG=5,
    WILSON_MEE_MEEDAG=6, KS_D=10, KS_DDAG=11, KS_DDDAG=12, KS_DDDAG_EE=13,
)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        d, i, p, u32, u64, l = C.c_double, C.c_int, C.c_void_p, C.c_uint32, C.c_uint64, C.c_long
        sig = {
            "clgo_philox4x32_10": (None, [p, p, p]),
            "clgo_gen_gauge_haar": (None, [p, u64, u32, p]),
            "clgo_gen_gauge_expH": (None, [p, u64, u32, d, p]),
            "clgo_gen_gauge_identity": (None, [p, p]),
            "clgo_gen_gauss": (None, [l, i, u64, u32, p]),
            "clgo_gen_z2": (None, [l, i, u64, u32, p]),
            "clgo_gen_z4": (None, [l, i, u64, u32, p]),
            "clgo_gen_point": (None, [l, i, l, i, p]),
            "clgo_zero_parity": (None, [p, i, i, p]),
            "clgo_plaquette": (d, [p, p]),
            "clgo_unitarity_deviation": (d, [l, p]),
            "clgo_bridgepp_to_clg": (None, [p, p, p]),
            "clgo_wilson_D": (None, [p, p, d, i, i, d, d, p, p]),
            "clgo_wilson_hop": (None, [p, p, i, i, p, p]),
            "clgo_wilson_mee": (None, [p, p, d, i, p, p, p]),
            "clgo_wilson_force": (None, [p, p, d, p, p, p]),
            "clgo_ks_D": (None, [p, p, d, i, i, d, d, p, p]),
            "clgo_ks_hop": (None, [p, p, i, p, p]),
            "clgo_ks_dddag_ee": (None, [p, p, d, p, p, p]),
            "clgo_ks_force": (None, [p, p, i, p, p, p, p]),
            "clgo_gamma": (i, [i, p, p, p]),
            "clgo_meson_correlator": (None, [p, p, i, p]),
            "clgo_condensate": (None, [l, p, p, i, p]),
            "clgo_op_len": (l, [p]),
            "clgo_apply": (None, [p, p, p]),
            "clgo_dot": (None, [l, p, p, p]),
            "clgo_norm2": (d, [l, p]),
            "clgo_axpy": (None, [l, d, d, p, p]),
            "clgo_gmres": (i, [p, p, p, p, i, i, d, i, p]),
            "clgo_bicgstab": (i, [p, p, p, p, i, i, i, d, i, d, i, p]),
            "clgo_cg": (i, [p, p, p, d, i, p]),
            "clgo_cgm": (i, [p, p, i, p, p, d, i, p]),
            "clgo_fom_ms": (i, [p, p, i, p, p, i, i, d, i, p]),
            "clgo_bicgstab_ms": (i, [p, p, i, p, p, i, i, d, i, p]),
            "clgo_gmres_ms": (i, [p, p, i, p, p, i, i, d, i, p]),
            "clgo_true_residual": (d, [p, p, p, d, d]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def _lat(L, bc=(1, 1, 1, -1)) -> Lat:
    return Lat((C.c_int * 4)(*L), (C.c_int * 4)(*bc))


def volume(L) -> int:
    return int(L[0]) * int(L[1]) * int(L[2]) * int(L[3])


def coords(L):
    """(V, 4) integer coordinates in CLG site order (t fastest)."""
    x, y, z, t = np.meshgrid(*[np.arange(n) for n in L], indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel(), t.ravel()], axis=1)


def parity_mask(L):
    return (coords(L).sum(axis=1) & 1).astype(np.int8)


# ------------------------------------------------------------------ fields
def gauge_haar(L, seed, field_id=1):
    U = np.empty((volume(L) * 4, 3, 3), np.complex128)
    lib().clgo_gen_gauge_haar(_ptr(np.asarray(L, np.int32)), seed, field_id, _ptr(U))
    return U


def gauge_expH(L, seed, eps, field_id=1):
    U = np.empty((volume(L) * 4, 3, 3), np.complex128)
    lib().clgo_gen_gauge_expH(_ptr(np.asarray(L, np.int32)), seed, field_id, eps, _ptr(U))
    return U


def gauge_identity(L):
    U = np.empty((volume(L) * 4, 3, 3), np.complex128)
    lib().clgo_gen_gauge_identity(_ptr(np.asarray(L, np.int32)), _ptr(U))
    return U


def gauss(nsites, ncomp, seed, field_id):
    psi = np.empty((nsites, ncomp), np.complex128)
    lib().clgo_gen_gauss(nsites, ncomp, seed, field_id, _ptr(psi))
    return psi


def z2(nsites, ncomp, seed, field_id):
    psi = np.empty((nsites, ncomp), np.complex128)
    lib().clgo_gen_z2(nsites, ncomp, seed, field_id, _ptr(psi))
    return psi


def z4(nsites, ncomp, seed, field_id):
    psi = np.empty((nsites, ncomp), np.complex128)
    lib().clgo_gen_z4(nsites, ncomp, seed, field_id, _ptr(psi))
    return psi


def philox(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().clgo_philox4x32_10(_ptr(c), _ptr(k), _ptr(o))
    return o


def plaquette(L, U):
    return lib().clgo_plaquette(_ptr(np.asarray(L, np.int32)), _ptr(np.ascontiguousarray(U)))


def unitarity_deviation(U):
    U = np.ascontiguousarray(U)
    return lib().clgo_unitarity_deviation(U.shape[0], _ptr(U))


def bridgepp_to_clg(L, bridge_reals):
    b = np.ascontiguousarray(bridge_reals, np.float64)
    U = np.empty((volume(L) * 4, 3, 3), np.complex128)
    lib().clgo_bridgepp_to_clg(_ptr(np.asarray(L, np.int32)), _ptr(b), _ptr(U))
    return U


# ------------------------------------------------------------------ operators
def wilson_D(L, U, psi, kappa, dagger=False, bc=(1, 1, 1, -1), coeff=None):
    psi = np.ascontiguousarray(psi, np.complex128)
    out = np.empty_like(psi)
    ct, cre, cim = 0, 0.0, 0.0
    if coeff is not None:
        if coeff == "minus":
            ct = 1
        elif isinstance(coeff, complex):
            ct, cre, cim = 3, coeff.real, coeff.imag
        else:
            ct, cre = 2, float(coeff)
    lat = _lat(L, bc)
    lib().clgo_wilson_D(C.byref(lat), _ptr(U), kappa, int(dagger), ct, cre, cim, _ptr(psi), _ptr(out))
    return out


def wilson_hop(L, U, psi, out_parity, dagger=False, bc=(1, 1, 1, -1)):
    psi = np.ascontiguousarray(psi, np.complex128)
    out = np.empty_like(psi)
    lat = _lat(L, bc)
    lib().clgo_wilson_hop(C.byref(lat), _ptr(U), int(dagger), out_parity, _ptr(psi), _ptr(out))
    return out


def wilson_mee(L, U, psi, kappa, dagger=False, bc=(1, 1, 1, -1)):
    psi = np.ascontiguousarray(psi, np.complex128)
    out = np.empty_like(psi)
    tmp = np.empty_like(psi)
    lat = _lat(L, bc)
    lib().clgo_wilson_mee(C.byref(lat), _ptr(U), kappa, int(dagger), _ptr(psi), _ptr(out), _ptr(tmp))
    return out


def wilson_force(L, U, X, Y, kappa, F=None, bc=(1, 1, 1, -1)):
    """F + the Wilson fermion force of X = (DD^+)^-1 phi, Y = D^+ X
    (_kernelDWilsonForceSU3, CFieldFermionWilsonSquareSU3.cu:170-231); F and U in
    the CLGBin link layout (V*4 links of 9 complex)."""
    X = np.ascontiguousarray(X, np.complex128)
    Y = np.ascontiguousarray(Y, np.complex128)
    out = np.zeros_like(np.ascontiguousarray(U, np.complex128)) if F is None else np.array(F, np.complex128)
    lat = _lat(L, bc)
    lib().clgo_wilson_force(C.byref(lat), _ptr(U), kappa, _ptr(X), _ptr(Y), _ptr(out))
    return out


GAMMAS = ["UNITY", "GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4", "GAMMA5", "GAMMA51", "GAMMA52", "GAMMA53", "GAMMA54",
          "GAMMA15", "GAMMA25", "GAMMA35", "GAMMA45", "SIGMA12", "SIGMA23", "SIGMA31", "SIGMA41", "SIGMA42", "SIGMA43",
          "SIGMA12E", "SIGMA23E", "SIGMA31E", "CHARGECONJG"]


def gamma(which):
    """(idx[4], z[4], next_symmetric_index) of EGammaMatrix `which` (chiral set)."""
    idx = (C.c_int * 4)()
    z = (C.c_int * 4)()
    ns = C.c_int()
    if lib().clgo_gamma(which, idx, z, C.byref(ns)) != 0:
        raise ValueError(which)
    return list(idx), list(z), ns.value


def gamma_matrix(which):
    idx, z, _ = gamma(which)
    m = np.zeros((4, 4), np.complex128)
    for r in range(4):
        m[r, idx[r]] = 1j ** z[r]
    return m


def meson_correlator(L, props, which):
    """C(t) of the 12 point-source propagators props[spin*3 + colour] (CMeasureMesonCorrelator.cu:26-174, 366-380)."""
    P = np.ascontiguousarray(np.stack([np.asarray(x, np.complex128).reshape(-1) for x in props]))
    assert P.shape[0] == 12
    out = np.zeros(L[3], np.float64)
    Li = (C.c_int * 4)(*L)
    lib().clgo_meson_correlator(Li, _ptr(P), which, _ptr(out))
    return out


def condensate(eta, psi, kind):
    """(1/V) sum_x eta^+ Gamma_kind psi (CMeasureChiralCondensate.cu:38-100, omega = 0)."""
    e = np.ascontiguousarray(eta, np.complex128).reshape(-1)
    q = np.ascontiguousarray(psi, np.complex128).reshape(-1)
    out = np.zeros(2, np.float64)
    lib().clgo_condensate(e.size // 12, _ptr(e), _ptr(q), kind, _ptr(out))
    return complex(out[0], out[1])


def ks_force(L, U, phi_i, phi_id, a, F=None, bc=(1, 1, 1, -1)):
    """F - the staggered rational force (_kernelDFermionKSForce,
    Staggered/CFieldFermionKSSU3.cu:216-262) of the fields phi_i[n] =
    (DD^+ + b_n)^-1 phi and phi_id[n] = D0 phi_i[n] with numerators a[n]."""
    pi = np.ascontiguousarray(np.stack([np.asarray(x, np.complex128).reshape(-1) for x in phi_i]))
    pd = np.ascontiguousarray(np.stack([np.asarray(x, np.complex128).reshape(-1) for x in phi_id]))
    aa = np.ascontiguousarray(a, np.float64)
    out = np.zeros_like(np.ascontiguousarray(U, np.complex128)) if F is None else np.array(F, np.complex128)
    lat = _lat(L, bc)
    lib().clgo_ks_force(C.byref(lat), _ptr(U), len(aa), _ptr(pi), _ptr(pd), _ptr(aa), _ptr(out))
    return out


def ks_D(L, U, chi, mass2am, dagger=False, bc=(1, 1, 1, -1), coeff=None):
    chi = np.ascontiguousarray(chi, np.complex128)
    out = np.empty_like(chi)
    ct, cre, cim = 0, 0.0, 0.0
    if coeff is not None:
        if coeff == "minus":
            ct = 1
        elif isinstance(coeff, complex):
            ct, cre, cim = 3, coeff.real, coeff.imag
        else:
            ct, cre = 2, float(coeff)
    lat = _lat(L, bc)
    lib().clgo_ks_D(C.byref(lat), _ptr(U), mass2am, int(dagger), ct, cre, cim, _ptr(chi), _ptr(out))
    return out


def ks_hop(L, U, chi, out_parity, bc=(1, 1, 1, -1)):
    chi = np.ascontiguousarray(chi, np.complex128)
    out = np.empty_like(chi)
    lat = _lat(L, bc)
    lib().clgo_ks_hop(C.byref(lat), _ptr(U), out_parity, _ptr(chi), _ptr(out))
    return out


def ks_dddag_ee(L, U, chi, mass2am, bc=(1, 1, 1, -1)):
    chi = np.ascontiguousarray(chi, np.complex128)
    out = np.empty_like(chi)
    tmp = np.empty_like(chi)
    lat = _lat(L, bc)
    lib().clgo_ks_dddag_ee(C.byref(lat), _ptr(U), mass2am, _ptr(chi), _ptr(out), _ptr(tmp))
    return out


class Operator:
    """An oracle operator (kind from ``OP``) with its scratch fields."""

    def __init__(self, kind, L, U, param, bc=(1, 1, 1, -1)):
        self.kind = OP[kind] if isinstance(kind, str) else kind
        self.L = tuple(L)
        self.U = np.ascontiguousarray(U, np.complex128)
        V = volume(L)
        shape = (V, 3) if self.kind >= 10 else (V, 4, 3)
        self.shape = shape
        self._tmp = np.zeros(shape, np.complex128)
        self._tmp2 = np.zeros(shape, np.complex128)
        self.op = Op(self.kind, _lat(L, bc), self.U.ctypes.data, param,
                     self._tmp.ctypes.data, self._tmp2.ctypes.data)

    def __call__(self, x):
        x = np.ascontiguousarray(x, np.complex128)
        out = np.empty_like(x)
        lib().clgo_apply(C.byref(self.op), _ptr(x), _ptr(out))
        return out

    def true_residual(self, b, x, shift=0j):
        return lib().clgo_true_residual(C.byref(self.op), _ptr(np.ascontiguousarray(b)),
                                        _ptr(np.ascontiguousarray(x)), shift.real, shift.imag)


def gmres(op: Operator, b, x0=None, maxdim=12, restart=100, accuracy=1e-20, absolute=False):
    b = np.ascontiguousarray(b, np.complex128)
    x = np.empty_like(b)
    info = Info()
    p0 = _ptr(np.ascontiguousarray(x0, np.complex128)) if x0 is not None else None
    lib().clgo_gmres(C.byref(op.op), _ptr(b), _ptr(x), p0, maxdim, restart, accuracy, int(absolute), C.byref(info))
    return x, info.as_dict()


def bicgstab(op: Operator, b, x0=None, dev_step=10, max_step=100, restart=10, accuracy=1e-20,
             absolute=False, small_rho=1e-30, std_omega=False):
    b = np.ascontiguousarray(b, np.complex128)
    x = np.empty_like(b)
    info = Info()
    p0 = _ptr(np.ascontiguousarray(x0, np.complex128)) if x0 is not None else None
    lib().clgo_bicgstab(C.byref(op.op), _ptr(b), _ptr(x), p0, dev_step, max_step, restart, accuracy,
                        int(absolute), small_rho, int(std_omega), C.byref(info))
    return x, info.as_dict()


def cg(op: Operator, b, tol=1e-10, maxiter=10000):
    b = np.ascontiguousarray(b, np.complex128)
    x = np.empty_like(b)
    info = Info()
    lib().clgo_cg(C.byref(op.op), _ptr(b), _ptr(x), tol, maxiter, C.byref(info))
    return x, info.as_dict()


def cgm(op: Operator, b, shifts, tol=1e-10, maxiter=10000):
    b = np.ascontiguousarray(b, np.complex128)
    sh = np.ascontiguousarray(shifts, np.float64)
    x = np.empty((len(sh),) + b.shape, np.complex128)
    info = Info()
    lib().clgo_cgm(C.byref(op.op), _ptr(b), len(sh), _ptr(sh), _ptr(x), tol, maxiter, C.byref(info))
    return x, info.as_dict()


def fom_ms(op: Operator, b, shifts, maxdim=12, restart=100, accuracy=1e-10, absolute=False):
    b = np.ascontiguousarray(b, np.complex128)
    sh = np.ascontiguousarray(np.asarray(shifts, np.complex128))
    x = np.empty((len(sh),) + b.shape, np.complex128)
    info = Info()
    lib().clgo_fom_ms(C.byref(op.op), _ptr(b), len(sh), _ptr(sh.view(np.float64)), _ptr(x), maxdim, restart,
                      accuracy, int(absolute), C.byref(info))
    return x, info.as_dict()


def gmres_ms(op: Operator, b, shifts, maxdim=10, restart=100, accuracy=1e-10, absolute=False):
    """CMultiShiftGMRES (CMultiShiftGMRES.cpp:113-330) restated: (A + c_n) x_n = b."""
    b = np.ascontiguousarray(b, np.complex128)
    sh = np.ascontiguousarray(np.asarray(shifts, np.complex128))
    x = np.empty((len(sh),) + b.shape, np.complex128)
    info = Info()
    lib().clgo_gmres_ms(C.byref(op.op), _ptr(b), len(sh), _ptr(sh.view(np.float64)), _ptr(x), maxdim, restart,
                        accuracy, int(absolute), C.byref(info))
    return x, info.as_dict()


def bicgstab_ms(op: Operator, b, shifts, dev_step=10, max_step=100, accuracy=1e-10, absolute=False):
    """CMultiShiftBiCGStab (CMultiShiftBiCGStab.cpp:73-437) restated: (A + c_n) x_n = b."""
    b = np.ascontiguousarray(b, np.complex128)
    sh = np.ascontiguousarray(np.asarray(shifts, np.complex128))
    x = np.empty((len(sh),) + b.shape, np.complex128)
    info = Info()
    lib().clgo_bicgstab_ms(C.byref(op.op), _ptr(b), len(sh), _ptr(sh.view(np.float64)), _ptr(x), dev_step, max_step,
                           accuracy, int(absolute), C.byref(info))
    return x, info.as_dict()


def dot(a, b):
    a = np.ascontiguousarray(a, np.complex128)
    b = np.ascontiguousarray(b, np.complex128)
    out = np.zeros(2)
    lib().clgo_dot(a.size, _ptr(a), _ptr(b), _ptr(out))
    return complex(out[0], out[1])
