"""B200-native fermion hot path of CLGLib (CudaLatticeGauge).

Python mirror of the reference's field / operator / solver interface over the
C ABI of ``libclgb200.so`` (include/clg_b200.h).  Class and method names follow
the reference (Code/CLGLib/...):

  CFieldGaugeSU3                 Data/Field/Gauge/CFieldGaugeSU3.h:18-121
  CFieldFermionWilsonSquareSU3   Data/Field/WilsonDirac/CFieldFermionWilsonSquareSU3.h
  CFieldFermionKSSU3             Data/Field/Staggered/CFieldFermionKSSU3.h
  CSLASolverGMRES / BiCGStab     SparseLinearAlgebra/CSolverGMRES.cpp, CSolverBiCGstab.cpp
  CMultiShiftCG / CMultiShiftFOM SparseLinearAlgebra/CMultiShiftSolver.h:38-47

Every device computation runs in the CUDA library; there is no Python or CPU
fallback: without the library or a B200 the calls raise CLGError.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libclgb200.so")

# ------------------------------------------------------------------ enums (include/clg_b200.h)
SUCCESS, ERR_BAD_ARG, ERR_CUDA, ERR_OOM, ERR_NOT_CONVERGED, ERR_BREAKDOWN, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_NO_DEVICE = range(9)

EFO_F_D, EFO_F_Ddagger, EFO_F_DDdagger, EFO_F_DD = 0, 1, 2, 3
OP_MEE, OP_MEE_DAG, OP_MEE_MEEDAG, OP_DEO, OP_DOE, OP_DDDAG_EE = 4, 5, 6, 7, 8, 9
EOCT_None, EOCT_Minus, EOCT_Real, EOCT_Complex = 0, 1, 2, 3
WILSON, STAGGERED = 0, 1
FULL, EVEN = 0, 1
DOUBLE, SINGLE, HALF = 0, 1, 2
LAYOUT_CLGBIN, LAYOUT_BRIDGEPP = 0, 1
GAUGE_IDENTITY, GAUGE_HAAR, GAUGE_EXPH, GAUGE_ZERO = 0, 1, 2, 3
# clg_file_format (EFieldFileType)
(FILE_CLGBIN_DOUBLE, FILE_CLGBIN_FLOAT, FILE_CLGBIN_COMPRESSED, FILE_CLGBIN_COMPRESSED_FLOAT, FILE_BRIDGEPP_BIN,
 FILE_BRIDGEPP_TXT) = range(6)
SOURCE_ZERO, SOURCE_GAUSS, SOURCE_Z2, SOURCE_POINT, SOURCE_Z4 = 0, 1, 2, 3, 4
(SOLVER_GMRES, SOLVER_BICGSTAB, SOLVER_CG, SOLVER_CGM, SOLVER_FOM_MS, SOLVER_GCRODR, SOLVER_NESTED_MS,
 SOLVER_BICGSTAB_MS, SOLVER_GMRESMDR, SOLVER_GMRES_MS) = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9
EEDT_SVD, EEDT_REV, EEDT_HEV = 0, 1, 2  # GCRO-DR deflation spaces (EEigenDeflationType)


class CLGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class SolverParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("max_dim", C.c_int32), ("restart", C.c_int32), ("accuracy", C.c_double),
        ("absolute_accuracy", C.c_int32), ("deviation_step", C.c_int32), ("max_step", C.c_int32),
        ("small_rho", C.c_double), ("inner_precision", C.c_int32), ("tol_true_rel", C.c_double),
        ("inner_tol", C.c_double), ("max_iterations", C.c_int32), ("max_outer", C.c_int32),
        ("even_odd", C.c_int32), ("use_graphs", C.c_int32), ("kdim", C.c_int32), ("deflation", C.c_int32),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32), ("outer", C.c_int32),
        ("true_rel_residual", C.c_double), ("seconds", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# (name, restype, argtypes) for every entry point of include/clg_b200.h
_P, _I, _D, _U64, _U32, _I64 = C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_uint32, C.c_int64
_S = C.c_int32
SIGNATURES = [
    ("clg_context_create", _S, [_I, _P, C.POINTER(_P)]),
    ("clg_context_destroy", _S, [_P]),
    ("clg_context_set_stream", _S, [_P, _P]),
    ("clg_context_synchronize", _S, [_P]),
    ("clg_status_string", C.c_char_p, [_S]),
    ("clg_last_error", C.c_char_p, [_P]),
    ("clg_context_kernel_count", _S, [_P, C.POINTER(_I64)]),
    ("clg_context_tuned", _S, [_P, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("clg_lattice_create", _S, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_P)]),
    ("clg_lattice_destroy", _S, [_P]),
    ("clg_gauge_create", _S, [_P, C.POINTER(_P)]),
    ("clg_gauge_destroy", _S, [_P]),
    ("clg_gauge_import", _S, [_P, _P, _I, _I]),
    ("clg_gauge_export", _S, [_P, _P, _I]),
    ("clg_gauge_random", _S, [_P, _I, _U64, _U32, _D]),
    ("clg_gauge_plaquette", _S, [_P, C.POINTER(_D)]),
    ("clg_gauge_unitarity", _S, [_P, C.POINTER(_D)]),
    ("clg_field_create", _S, [_P, _I, _I, _I, _I, _D, C.POINTER(_P)]),
    ("clg_field_destroy", _S, [_P]),
    ("clg_field_set_param", _S, [_P, _D]),
    ("clg_field_import", _S, [_P, _I, _P, _I]),
    ("clg_field_export", _S, [_P, _I, _P, _I]),
    ("clg_field_import_async", _S, [_P, _I, _P]),
    ("clg_field_export_async", _S, [_P, _I, _P]),
    ("clg_field_wait", _S, [_P]),
    ("clg_field_random", _S, [_P, _I, _I, _U64, _U32, _I64, _I]),
    ("clg_field_copy", _S, [_P, _P]),
    ("clg_apply", _S, [_I, _P, _P, _I, _D, _D]),
    ("clg_apply_to", _S, [_I, _P, _P, _P, _I, _D, _D]),
    ("clg_dot", _S, [_P, _P, _P]),
    ("clg_dot_noalloc", _S, [_P, _P, _P]),
    ("clg_norm2", _S, [_P, _P]),
    ("clg_axpy", _S, [_P, _D, _D, _P]),
    ("clg_scale", _S, [_P, _D, _D]),
    ("clg_zero", _S, [_P]),
    ("clg_solver_default_params", _S, [_I, C.POINTER(SolverParams)]),
    ("clg_solver_create", _S, [_P, C.POINTER(SolverParams), C.POINTER(_P)]),
    ("clg_solver_destroy", _S, [_P]),
    ("clg_solver_reset", _S, [_P]),
    ("clg_solve", _S, [_P, _P, _P, _P, _I, _P, _P]),
    ("clg_solve_multishift", _S, [_P, _P, _I, _P, _P, _P, _I, _P]),
    ("clg_solve_lattices", _S, [_P, _I, _P, _P, _P, _I, _P]),
    ("clg_rational_apply", _S, [_P, _P, _P, _I, _I, _D, _P, _P, _P]),
    ("clg_gauge_load", _S, [_P, C.c_char_p, _I]),
    ("clg_gauge_save", _S, [_P, C.c_char_p, _I, C.c_char_p]),
    ("clg_md5", _S, [_P, C.c_size_t, C.c_char_p]),
    ("clg_field_save", _S, [_P, _I, C.c_char_p, _I, C.c_char_p]),
    ("clg_field_load", _S, [_P, _I, C.c_char_p, _I]),
    ("clg_wilson_force", _S, [_P, _P, _P, _P]),
    ("clg_wilson_fermion_force", _S, [_P, _P, _P, _P, _P, _P]),
    ("clg_ks_force", _S, [_P, _P, _I, _P, _P, _P]),
    ("clg_ks_fermion_force", _S, [_P, _P, _P, _P, _I, _P, _P, _P]),
    ("clg_small_eig", _S, [_I, _P, _P, _P, _P]),
    ("clg_meson_correlator", _S, [_P, _P, _P, _I, _P, _P, _P]),
    ("clg_meson_contract", _S, [_P, _I, _P, _P]),
    ("clg_chiral_condensate", _S, [_P, _P, _P, _P, C.c_uint64, _P, _P]),
    ("clg_condensate_contract", _S, [_P, _P, _P]),
]

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libclgb200.so (raises CLGError if it is missing: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CLGError(ERR_NO_DEVICE, f"{path} is missing; build it with `python -m cudalatticegauge_b200.build`")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


class Context:
    """CUDA device + stream that owns every object created from it."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.clg_context_create(device, C.c_void_p(stream) if stream else None, C.byref(h))
        if st != SUCCESS:
            raise CLGError(st, f"clg_context_create: {self.lib.clg_status_string(st).decode()}")
        self.h = h

    def check(self, st: int, what: str):
        if st != SUCCESS:
            raise CLGError(st, f"{what}: {self.lib.clg_status_string(st).decode()}: {self.lib.clg_last_error(self.h).decode()}")

    def synchronize(self):
        self.check(self.lib.clg_context_synchronize(self.h), "synchronize")

    def set_stream(self, stream: Optional[int]):
        self.check(self.lib.clg_context_set_stream(self.h, C.c_void_p(stream) if stream else None), "set_stream")

    def kernel_count(self) -> int:
        n = C.c_int64()
        self.check(self.lib.clg_context_kernel_count(self.h, C.byref(n)), "kernel_count")
        return n.value

    def tuned(self) -> dict:
        """The autotuner's choices: kernel key -> (block size, variant)."""
        need = C.c_size_t()
        self.check(self.lib.clg_context_tuned(self.h, None, 0, C.byref(need)), "clg_context_tuned")
        buf = C.create_string_buffer(need.value + 1)
        self.check(self.lib.clg_context_tuned(self.h, buf, need.value + 1, C.byref(need)), "clg_context_tuned")
        out = {}
        for line in buf.value.decode().splitlines():
            k, v = line.rsplit("=", 1)
            out[k] = (int(v) & 0xFFFF, int(v) >> 16)
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.clg_context_destroy(self.h)
            self.h = None


class Lattice:
    def __init__(self, ctx: Context, dims: Sequence[int], fermion_bc: Sequence[int] = (1, 1, 1, -1)):
        self.ctx, self.dims, self.bc = ctx, tuple(int(d) for d in dims), tuple(int(b) for b in fermion_bc)
        h = C.c_void_p()
        ctx.check(ctx.lib.clg_lattice_create(ctx.h, (C.c_int * 4)(*self.dims), (C.c_int * 4)(*self.bc), C.byref(h)),
                  "clg_lattice_create")
        self.h = h
        self.volume = int(np.prod(self.dims))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.clg_lattice_destroy(self.h)
            self.h = None


class CFieldGaugeSU3:
    """SU(3) gauge field (Data/Field/Gauge/CFieldGaugeSU3.h:18-121)."""

    def __init__(self, lattice: Lattice):
        self.lat, self.ctx = lattice, lattice.ctx
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.clg_gauge_create(lattice.h, C.byref(h)), "clg_gauge_create")
        self.h = h

    def InitialField(self, kind: int, seed: int = 0, field_id: int = 1, eps: float = 0.0):
        self.ctx.check(self.ctx.lib.clg_gauge_random(self.h, kind, seed, field_id, eps), "clg_gauge_random")

    def InitialWithByte(self, links: np.ndarray, layout: int = LAYOUT_CLGBIN):
        """links: complex128 [V*4, 3, 3] (or float64 raw 18 reals per link) in CLGBin or Bridge++ order."""
        a = np.ascontiguousarray(links)
        if a.dtype == np.complex128:
            a = a.view(np.float64)
        a = np.ascontiguousarray(a, np.float64)
        if a.size != self.lat.volume * 4 * 18:
            raise CLGError(ERR_BAD_ARG, "gauge data has the wrong size")
        self.ctx.check(self.ctx.lib.clg_gauge_import(self.h, _ptr(a), layout, 0), "clg_gauge_import")

    def CopyDataOut(self) -> np.ndarray:
        out = np.empty((self.lat.volume * 4, 3, 3), np.complex128)
        self.ctx.check(self.ctx.lib.clg_gauge_export(self.h, _ptr(out), 0), "clg_gauge_export")
        return out

    def InitialFieldWithFile(self, path: str, fmt: int = FILE_CLGBIN_DOUBLE):
        """CFieldGaugeSU3::InitialFieldWithFile (CFieldGaugeSU3.cu:1080-1265)."""
        self.ctx.check(self.ctx.lib.clg_gauge_load(self.h, os.fsencode(path), fmt), "clg_gauge_load")

    def SaveToFile(self, path: str, fmt: int = FILE_CLGBIN_DOUBLE) -> str:
        """CField::SaveToFile / SaveToCompressedFile; returns the MD5 of the bytes written."""
        out = C.create_string_buffer(33)
        self.ctx.check(self.ctx.lib.clg_gauge_save(self.h, os.fsencode(path), fmt, out), "clg_gauge_save")
        return out.value.decode()

    def plaquette(self) -> float:
        v = C.c_double()
        self.ctx.check(self.ctx.lib.clg_gauge_plaquette(self.h, C.byref(v)), "clg_gauge_plaquette")
        return v.value

    def unitarity(self) -> float:
        v = C.c_double()
        self.ctx.check(self.ctx.lib.clg_gauge_unitarity(self.h, C.byref(v)), "clg_gauge_unitarity")
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.clg_gauge_destroy(self.h)
            self.h = None


class _FermionField:
    KIND = WILSON
    NC = 12

    def __init__(self, lattice: Lattice, param: float, subset: int = FULL, precision: int = DOUBLE, nrhs: int = 1):
        self.lat, self.ctx = lattice, lattice.ctx
        self.subset, self.precision, self.nrhs, self.param = subset, precision, nrhs, param
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.clg_field_create(lattice.h, self.KIND, subset, precision, nrhs, param, C.byref(h)),
                       "clg_field_create")
        self.h = h

    # ------------------------------------------------------------ data movement (CLGBin order)
    def _shape(self):
        return (self.lat.volume, 4, 3) if self.NC == 12 else (self.lat.volume, 3)

    def from_numpy(self, data: np.ndarray, rhs: int = 0):
        a = np.ascontiguousarray(data, np.complex128)
        if a.size != self.lat.volume * self.NC:
            raise CLGError(ERR_BAD_ARG, "field data has the wrong size")
        self.ctx.check(self.ctx.lib.clg_field_import(self.h, rhs, _ptr(a), 0), "clg_field_import")

    def to_numpy(self, rhs: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self._shape(), np.complex128)
        elif out.dtype != np.complex128 or out.size != self.lat.volume * self.NC or not out.flags["C_CONTIGUOUS"]:
            raise CLGError(ERR_BAD_ARG, "export buffer has the wrong size or type")
        self.ctx.check(self.ctx.lib.clg_field_export(self.h, rhs, _ptr(out), 0), "clg_field_export")
        return out

    # asynchronous transfers (clg_field_import_async / export_async / wait): the
    # arrays should be pinned (e.g. torch.empty(..., pin_memory=True).numpy())
    # and are kept alive here until wait()
    def from_numpy_async(self, data: np.ndarray, rhs: int = 0):
        if data.dtype != np.complex128 or data.size != self.lat.volume * self.NC or not data.flags["C_CONTIGUOUS"]:
            raise CLGError(ERR_BAD_ARG, "import buffer has the wrong size or type")
        self.ctx.check(self.ctx.lib.clg_field_import_async(self.h, rhs, _ptr(data)), "clg_field_import_async")
        self._inflight = getattr(self, "_inflight", []) + [data]

    def to_numpy_async(self, out: np.ndarray, rhs: int = 0):
        if out.dtype != np.complex128 or out.size != self.lat.volume * self.NC or not out.flags["C_CONTIGUOUS"]:
            raise CLGError(ERR_BAD_ARG, "export buffer has the wrong size or type")
        self.ctx.check(self.ctx.lib.clg_field_export_async(self.h, rhs, _ptr(out)), "clg_field_export_async")
        self._inflight = getattr(self, "_inflight", []) + [out]

    def wait(self):
        self.ctx.check(self.ctx.lib.clg_field_wait(self.h), "clg_field_wait")
        self._inflight = []

    def InitialFieldWithFile(self, path: str, fmt: int = FILE_CLGBIN_DOUBLE, rhs: int = 0):
        """InitialFieldWithFile for a fermion field: CLGBin double or float."""
        self.ctx.check(self.ctx.lib.clg_field_load(self.h, rhs, os.fsencode(path), fmt), "clg_field_load")

    def SaveToFile(self, path: str, fmt: int = FILE_CLGBIN_DOUBLE, rhs: int = 0) -> str:
        """CField::SaveToFile for one right-hand side; returns the MD5 of the bytes written."""
        out = C.create_string_buffer(33)
        self.ctx.check(self.ctx.lib.clg_field_save(self.h, rhs, os.fsencode(path), fmt, out), "clg_field_save")
        return out.value.decode()

    def InitialField(self, kind: int, seed: int = 0, field_id: int = 2, rhs: int = 0, site: int = 0, comp: int = 0):
        self.ctx.check(self.ctx.lib.clg_field_random(self.h, rhs, kind, seed, field_id, site, comp), "clg_field_random")

    def InitialAsSource(self, site: int, comp: int, rhs: int = 0):
        self.InitialField(SOURCE_POINT, rhs=rhs, site=site, comp=comp)

    # ------------------------------------------------------------ operators (CField::ApplyOperator)
    def ApplyOperator(self, op: int, gauge: CFieldGaugeSU3, coeff_type: int = EOCT_None, cre: float = 1.0,
                      cim: float = 0.0):
        self.ctx.check(self.ctx.lib.clg_apply(op, self.h, gauge.h, coeff_type, cre, cim), "clg_apply")

    def apply_to(self, op: int, out: "_FermionField", gauge: CFieldGaugeSU3, coeff_type: int = EOCT_None,
                 cre: float = 1.0, cim: float = 0.0):
        self.ctx.check(self.ctx.lib.clg_apply_to(op, out.h, self.h, gauge.h, coeff_type, cre, cim), "clg_apply_to")

    def D(self, gauge, coeff_type=EOCT_None, cre=1.0, cim=0.0):
        self.ApplyOperator(EFO_F_D, gauge, coeff_type, cre, cim)

    def Ddagger(self, gauge, coeff_type=EOCT_None, cre=1.0, cim=0.0):
        self.ApplyOperator(EFO_F_Ddagger, gauge, coeff_type, cre, cim)

    def DDdagger(self, gauge, coeff_type=EOCT_None, cre=1.0, cim=0.0):
        self.ApplyOperator(EFO_F_DDdagger, gauge, coeff_type, cre, cim)

    # ------------------------------------------------------------ BLAS (CField.h:127-201)
    def Dot(self, other: "_FermionField"):
        out = np.zeros(2 * self.nrhs)
        self.ctx.check(self.ctx.lib.clg_dot(self.h, other.h, _ptr(out)), "clg_dot")
        z = out[0::2] + 1j * out[1::2]
        return z[0] if self.nrhs == 1 else z

    def norm2(self):
        out = np.zeros(self.nrhs)
        self.ctx.check(self.ctx.lib.clg_norm2(self.h, _ptr(out)), "clg_norm2")
        return out[0] if self.nrhs == 1 else out

    def Axpy(self, a, other: "_FermionField"):
        a = complex(a)
        self.ctx.check(self.ctx.lib.clg_axpy(self.h, a.real, a.imag, other.h), "clg_axpy")

    def AxpyPlus(self, other):
        self.Axpy(1.0, other)

    def AxpyMinus(self, other):
        self.Axpy(-1.0, other)

    def ScalarMultply(self, a):
        a = complex(a)
        self.ctx.check(self.ctx.lib.clg_scale(self.h, a.real, a.imag), "clg_scale")

    def Zero(self):
        self.ctx.check(self.ctx.lib.clg_zero(self.h), "clg_zero")

    def CopyTo(self, other: "_FermionField"):
        self.ctx.check(self.ctx.lib.clg_field_copy(other.h, self.h), "clg_field_copy")

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.clg_field_destroy(self.h)
            self.h = None


class CFieldFermionWilsonSquareSU3(_FermionField):
    """Wilson fermion, param = Hopping (kappa)."""
    KIND, NC = WILSON, 12

    @staticmethod
    def DerivateDOperator(force: CFieldGaugeSU3, dphi: "CFieldFermionWilsonSquareSU3",
                          dddphi: "CFieldFermionWilsonSquareSU3", gauge: CFieldGaugeSU3):
        """force += the Wilson fermion force from X = dddphi = (DD^+)^-1 phi and
        Y = dphi = D^+ X (CFieldFermionWilsonSquareSU3.cu:260-275, argument order
        as there: force, D^+ X, X, gauge)."""
        gauge.ctx.check(gauge.ctx.lib.clg_wilson_force(force.h, gauge.h, dddphi.h, dphi.h), "clg_wilson_force")

    def CalculateForceS(self, gauge: CFieldGaugeSU3, force: CFieldGaugeSU3, solver: "_Solver",
                        cache: Optional["CFieldFermionWilsonSquareSU3"] = None):
        """force += the force of the pseudofermion action phi^+ (DD^+)^-1 phi, phi = self
        (CFieldFermionWilsonSquareSU3.cu:1016-1100).  cache (nullable) is the start
        vector of the D D^+ solve and receives its solution.  Returns the solve infos."""
        infos = (SolveInfo * self.nrhs)()
        st = self.ctx.lib.clg_wilson_fermion_force(solver.h, force.h, gauge.h, self.h, cache.h if cache else None, infos)
        self.ctx.check(st, "clg_wilson_fermion_force")
        return [i.as_dict() for i in infos]


class CFieldFermionKSSU3(_FermionField):
    """Staggered (Kogut-Susskind) fermion, param = Mass (= 2am)."""
    KIND, NC = STAGGERED, 3

    @staticmethod
    def DerivateD0(force: CFieldGaugeSU3, gauge: CFieldGaugeSU3, phi_i: Sequence["CFieldFermionKSSU3"],
                   phi_id: Sequence["CFieldFermionKSSU3"], numerators: Sequence[float]):
        """force -= the staggered rational force of phi_i = (DD^+ + b_i)^-1 phi and
        phi_id = D0 phi_i with the given numerators (CFieldFermionKSSU3.cu:216-262, :316-331)."""
        n = len(numerators)
        if len(phi_i) != n or len(phi_id) != n:
            raise CLGError(ERR_BAD_ARG, "one phi_i and one phi_id per numerator")
        hi = (C.c_void_p * n)(*[f.h.value for f in phi_i])
        hd = (C.c_void_p * n)(*[f.h.value for f in phi_id])
        a = np.ascontiguousarray(numerators, np.float64)
        gauge.ctx.check(gauge.ctx.lib.clg_ks_force(force.h, gauge.h, n, hi, hd, _ptr(a)), "clg_ks_force")

    def CalculateForceS(self, gauge: CFieldGaugeSU3, force: CFieldGaugeSU3, solver: "_Solver",
                        numerators: Sequence[float], shifts: Sequence[float]):
        """force += the force of the rational pseudofermion action (the reference's
        m_rMD: numerators a_i, shifts b_i), phi = self (CFieldFermionKSSU3.cu:412-500).
        solver is a CMultiShiftCG (or CMultiShiftFOM).  Returns the solve infos."""
        a = np.ascontiguousarray(numerators, np.float64)
        b = np.ascontiguousarray(shifts, np.float64)
        if a.size != b.size:
            raise CLGError(ERR_BAD_ARG, "one shift per numerator")
        infos = (SolveInfo * a.size)()
        st = self.ctx.lib.clg_ks_fermion_force(solver.h, force.h, gauge.h, self.h, a.size, _ptr(a), _ptr(b), infos)
        self.ctx.check(st, "clg_ks_fermion_force")
        return [i.as_dict() for i in infos]


class _Solver:
    KIND = SOLVER_GMRES

    def __init__(self, ctx: Context, **kw):
        self.ctx = ctx
        p = SolverParams()
        ctx.check(ctx.lib.clg_solver_default_params(self.KIND, C.byref(p)), "clg_solver_default_params")
        names = {
            "MaxDim": "max_dim", "MDim": "max_dim", "KDim": "kdim", "DeflateSpace": "deflation", "Restart": "restart", "Accuracy": "accuracy", "AbsoluteAccuracy": "absolute_accuracy",
            "DiviationStep": "deviation_step", "MaxStep": "max_step", "SmallRho": "small_rho",
        }
        for k, v in kw.items():
            setattr(p, names.get(k, k), v)
        self.params = p
        h = C.c_void_p()
        ctx.check(ctx.lib.clg_solver_create(ctx.h, C.byref(p), C.byref(h)), "clg_solver_create")
        self.h = h

    def Solve(self, x: _FermionField, b: _FermionField, gauge: CFieldGaugeSU3, op: int = EFO_F_D,
              start: Optional[_FermionField] = None, raise_on_fail: bool = True):
        infos = (SolveInfo * b.nrhs)()
        st = self.ctx.lib.clg_solve(self.h, x.h, b.h, gauge.h, op, start.h if start else None, infos)
        out = [i.as_dict() for i in infos]
        if st != SUCCESS and raise_on_fail:
            self.ctx.check(st, "clg_solve")
        return out

    def SolveLattices(self, xs: Sequence["_FermionField"], bs: Sequence["_FermionField"],
                      gauges: Sequence[CFieldGaugeSU3], op: int = EFO_F_D, raise_on_fail: bool = True):
        """clg_solve_lattices: b[i] on lattice i (gauge gauges[i]) solved together in one
        solve; returns one info dict per right-hand side, in lattice order."""
        n = len(bs)
        xa = (C.c_void_p * n)(*[x.h.value for x in xs])
        ba = (C.c_void_p * n)(*[b.h.value for b in bs])
        ua = (C.c_void_p * n)(*[u.h.value for u in gauges])
        infos = (SolveInfo * sum(b.nrhs for b in bs))()
        st = self.ctx.lib.clg_solve_lattices(self.h, n, xa, ba, ua, op, infos)
        out = [i.as_dict() for i in infos]
        if st != SUCCESS and raise_on_fail:
            self.ctx.check(st, "clg_solve_lattices")
        return out

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.clg_solver_destroy(self.h)
            self.h = None


class CSLASolverGMRES(_Solver):
    KIND = SOLVER_GMRES


class CSLASolverBiCGStab(_Solver):
    KIND = SOLVER_BICGSTAB


class CSLASolverCG(_Solver):
    KIND = SOLVER_CG


class _MultiShift(_Solver):
    def Solve(self, xs: Sequence[_FermionField], shifts: Sequence[complex], b: _FermionField, gauge: CFieldGaugeSU3,
              op: int = EFO_F_DDdagger, raise_on_fail: bool = True):
        n = len(shifts)
        arr = (C.c_void_p * n)(*[x.h.value for x in xs])
        sh = np.ascontiguousarray(np.asarray(shifts, np.complex128).view(np.float64))
        infos = (SolveInfo * n)()
        st = self.ctx.lib.clg_solve_multishift(self.h, arr, n, _ptr(sh), b.h, gauge.h, op, infos)
        out = [i.as_dict() for i in infos]
        if st != SUCCESS and raise_on_fail:
            self.ctx.check(st, "clg_solve_multishift")
        return out

    def rational(self, f: _FermionField, gauge: CFieldGaugeSU3, op: int, c: float, a: Sequence[float],
                 b: Sequence[float]):
        """CFieldFermion::RationalApproximation: f <- c f + sum_i a_i (op + b_i)^-1 f."""
        deg = len(a)
        aa = np.ascontiguousarray(a, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        infos = (SolveInfo * deg)()
        st = self.ctx.lib.clg_rational_apply(self.h, f.h, gauge.h, op, deg, c, _ptr(aa), _ptr(bb), infos)
        self.ctx.check(st, "clg_rational_apply")
        return [i.as_dict() for i in infos]


class CMultiShiftCG(_MultiShift):
    KIND = SOLVER_CGM


class CMultiShiftFOM(_MultiShift):
    """CMultiShiftFOM (CMultiShiftFOM.cpp:97-270): restarted FOM(MaxDim <= 32)
    over one Krylov space for every shift, FP64 fields; MaxDim 30 as the
    reference's TestSuit_Solver.yaml blocks use."""
    KIND = SOLVER_FOM_MS

    def __init__(self, ctx: Context, **kw):
        kw.setdefault("MaxDim", 30)
        super().__init__(ctx, **kw)


class CMultiShiftGMRES(_MultiShift):
    """CMultiShiftGMRES (CMultiShiftGMRES.cpp:113-330): restarted GMRES on the seed
    system, every shift's residual collinear with the seed's; FP64 fields."""
    KIND = SOLVER_GMRES_MS

    def __init__(self, ctx: Context, **kw):
        kw.setdefault("MaxDim", 10)
        super().__init__(ctx, **kw)


class CMultiShiftBiCGStab(_MultiShift):
    """CMultiShiftBiCGStab (CMultiShiftBiCGStab.cpp:73-437): BiCGStab-M over one
    Krylov space for every shift, FP64 fields; DiviationStep / MaxStep as the
    reference's keys."""
    KIND = SOLVER_BICGSTAB_MS


class CMultiShiftNested(_MultiShift):
    """CMultiShiftNested (CMultiShiftNested.cpp:69-145) in batched form: every
    shift one right-hand side of a shifted solve (no shared Krylov space)."""
    KIND = SOLVER_NESTED_MS


class CSLASolverGCRODR(_Solver):
    """GCRO-DR with a recycled subspace kept between solves (CSolverGCRODR.cpp);
    MDim / KDim as the reference's keys, FP64, one right-hand side."""
    KIND = SOLVER_GCRODR

    def Reset(self):
        """Drop the recycled subspace (the start of a new trajectory)."""
        self.ctx.check(self.ctx.lib.clg_solver_reset(self.h), "clg_solver_reset")


class CSLASolverGMRESMDR(CSLASolverGCRODR):
    """GMRES-MDR (CSolverGMRESMDR.cpp:16-170): GCRO-DR whose solves from a kept
    U_k start by rotating it to the deflation problem's eigenvectors."""
    KIND = SOLVER_GMRESMDR


# EGammaMatrix (clg_gamma)
GAMMAS = ["UNITY", "GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4", "GAMMA5", "GAMMA51", "GAMMA52", "GAMMA53", "GAMMA54",
          "GAMMA15", "GAMMA25", "GAMMA35", "GAMMA45", "SIGMA12", "SIGMA23", "SIGMA31", "SIGMA41", "SIGMA42", "SIGMA43",
          "SIGMA12E", "SIGMA23E", "SIGMA31E", "CHARGECONJG"]


def _gamma_ids(gammas):
    return np.ascontiguousarray([GAMMAS.index(g) if isinstance(g, str) else int(g) for g in gammas], np.int32)


class CMeasureMesonCorrelator:
    """Meson correlator of the 12 point-source propagators at the origin
    (Measurement/CMeasureMesonCorrelator.cu): Calculate() solves them in one
    batched call and returns {gamma: C(t)}; the running average over
    configurations is kept as the reference's m_lstResults."""

    def __init__(self, solver: "_Solver", lattice: Lattice, kappa: float, gammas=("UNITY",)):
        self.solver, self.lat, self.kappa = solver, lattice, kappa
        self.gammas = list(gammas)
        self.prop = CFieldFermionWilsonSquareSU3(lattice, kappa, nrhs=12)
        self.results = None
        self.count = 0

    def contract(self, prop: "CFieldFermionWilsonSquareSU3") -> dict:
        ids = _gamma_ids(self.gammas)
        out = np.zeros((len(ids), self.lat.dims[3]), np.float64)
        self.lat.ctx.check(self.lat.ctx.lib.clg_meson_contract(prop.h, len(ids), _ptr(ids), _ptr(out)),
                           "clg_meson_contract")
        return {g: out[k] for k, g in enumerate(self.gammas)}

    def Calculate(self, gauge: CFieldGaugeSU3):
        ids = _gamma_ids(self.gammas)
        out = np.zeros((len(ids), self.lat.dims[3]), np.float64)
        infos = (SolveInfo * 12)()
        st = self.lat.ctx.lib.clg_meson_correlator(self.solver.h, gauge.h, self.prop.h, len(ids), _ptr(ids), _ptr(out),
                                                   infos)
        self.lat.ctx.check(st, "clg_meson_correlator")
        self.results = out if self.results is None else (self.results * self.count + out) / (self.count + 1)
        self.count += 1
        return {g: out[k] for k, g in enumerate(self.gammas)}, [i.as_dict() for i in infos]


class CMeasureChiralCondensate:
    """Z4-noise condensate traces (Measurement/CMeasureChiralCondensate.cu):
    Calculate() draws `fields` Z4 noise vectors, solves them in one batched call
    and returns the nine traces (1, gamma1..gamma5, gamma4 gamma5, gamma1, gamma2)
    averaged over the noise vectors."""

    def __init__(self, solver: "_Solver", lattice: Lattice, kappa: float, fields: int = 8):
        self.solver, self.lat = solver, lattice
        self.eta = CFieldFermionWilsonSquareSU3(lattice, kappa, nrhs=fields)
        self.psi = CFieldFermionWilsonSquareSU3(lattice, kappa, nrhs=fields)

    def Calculate(self, gauge: CFieldGaugeSU3, seed: int = 0):
        out = np.zeros(18, np.float64)
        infos = (SolveInfo * self.eta.nrhs)()
        st = self.lat.ctx.lib.clg_chiral_condensate(self.solver.h, gauge.h, self.eta.h, self.psi.h, seed, _ptr(out),
                                                    infos)
        self.lat.ctx.check(st, "clg_chiral_condensate")
        return out[0::2] + 1j * out[1::2], [i.as_dict() for i in infos]

    @staticmethod
    def contract(eta: "CFieldFermionWilsonSquareSU3", psi: "CFieldFermionWilsonSquareSU3") -> np.ndarray:
        """per right-hand side r and kind k: (1/V) sum_x eta_r^+ Gamma_k psi_r, shape (nrhs, 9) complex"""
        out = np.zeros(eta.nrhs * 18, np.float64)
        eta.ctx.check(eta.ctx.lib.clg_condensate_contract(eta.h, psi.h, _ptr(out)), "clg_condensate_contract")
        return (out[0::2] + 1j * out[1::2]).reshape(eta.nrhs, 9)


def small_eig(A: np.ndarray, B: Optional[np.ndarray] = None):
    """Eigenvalues and unit eigenvectors (columns) of A, or of A x = w B x (clg_small_eig)."""
    n = A.shape[0]
    a = np.ascontiguousarray(A, np.complex128)
    b = None if B is None else np.ascontiguousarray(B, np.complex128)
    w = np.zeros(n, np.complex128)
    x = np.zeros((n, n), np.complex128)
    st = load_library().clg_small_eig(n, _ptr(a), None if b is None else _ptr(b), _ptr(w), _ptr(x))
    if st != SUCCESS:
        raise CLGError(st, "clg_small_eig")
    return w, x


def md5(data) -> str:
    """CLGMD5Hash of a bytes-like object through the library (RFC 1321)."""
    b = bytes(data)
    out = C.create_string_buffer(33)
    st = load_library().clg_md5(b, len(b), out)
    if st != SUCCESS:
        raise CLGError(st, "clg_md5")
    return out.value.decode()


def eo_parity(dims) -> np.ndarray:
    """Parity (x+y+z+t)&1 of every site in CLG order."""
    x, y, z, t = np.meshgrid(*[np.arange(n) for n in dims], indexing="ij")
    return ((x + y + z + t) & 1).ravel()
