/*
 * clg_b200.h -- C ABI of the B200 (sm_100a) fermion hot path of CLGLib.
 *
 * Drop-in boundary for CLGLib's Wilson / staggered Dirac operators and the
 * Krylov solvers that apply them.  Each entry point names the reference
 * interface it replaces (paths relative to the CudaLatticeGauge tree,
 * Code/CLGLib/...).  Plain C types only: opaque handles, pointers, sizes.
 *
 * Conventions shared with the reference (CLGBin order):
 *   site   s = ((x*Ly + y)*Lz + z)*Lt + t                  Data/CCommonData.h:274-277
 *   link   l = s*4 + mu (mu = x,y,z,t), 18 reals row-major  Data/Field/Gauge/CFieldGaugeSU3.cu:1199-1222
 *   Wilson spinor: 24 reals per site, spin-major then colour Tools/Math/Vectors.h:575-888
 *   staggered vector: 6 reals per site                      Tools/Math/Vectors.h:287-571
 *
 * Every call returns a clg_status; nothing exits or aborts the process (the
 * reference exits on CUDA errors, Core/CudaHelperFunctions.h:1264-1275).
 * All device work of a context is ordered on the context's CUDA stream.
 */
#ifndef CLG_B200_H
#define CLG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef int32_t clg_status;
enum {
    CLG_SUCCESS = 0,
    CLG_ERR_BAD_ARG = 1,        /* invalid handle, size or option                       */
    CLG_ERR_CUDA = 2,           /* a CUDA runtime call failed (see clg_last_error)       */
    CLG_ERR_OOM = 3,            /* device allocation failed                              */
    CLG_ERR_NOT_CONVERGED = 4,  /* solver reached its iteration limit (reference: FALSE)  */
    CLG_ERR_BREAKDOWN = 5,      /* Krylov breakdown (rho ~ 0, NaN/Inf)                   */
    CLG_ERR_TIMEOUT = 6,        /* a bounded device wait ran out                         */
    CLG_ERR_UNSUPPORTED = 7,    /* combination not implemented (e.g. odd extents)        */
    CLG_ERR_NO_DEVICE = 8       /* no CUDA device / not an sm_100 device                  */
};

/* ------------------------------------------------------------------ enums */
/* EFieldOperator (Data/Field/CField.h:37-56) plus the even-odd forms of
 * Docs/SparseLinearAlgebra/evenodd.tex:11-16 */
typedef enum {
    CLG_OP_D = 0,            /* EFO_F_D                                           */
    CLG_OP_DDAG = 1,         /* EFO_F_Ddagger                                     */
    CLG_OP_DDDAG = 2,        /* EFO_F_DDdagger : D (D^+ x)                        */
    CLG_OP_DD = 3,           /* EFO_F_DD                                          */
    CLG_OP_MEE = 4,          /* Wilson: 1 - k^2 H_eo H_oe on even sites            */
    CLG_OP_MEE_DAG = 5,      /* Wilson: 1 - k^2 H^+_eo H^+_oe                      */
    CLG_OP_MEE_MEEDAG = 6,   /* Wilson: M_ee M_ee^+                               */
    CLG_OP_DEO = 7,          /* hopping even <- odd (no kappa / mass)              */
    CLG_OP_DOE = 8,          /* hopping odd <- even                                */
    CLG_OP_DDDAG_EE = 9      /* staggered: (2am)^2 - H_eo H_oe on even sites       */
} clg_op;

/* EOperatorCoefficientType (Data/Field/CField.h:62-68) */
typedef enum { CLG_COEFF_NONE = 0, CLG_COEFF_MINUS = 1, CLG_COEFF_REAL = 2, CLG_COEFF_COMPLEX = 3 } clg_coeff;

typedef enum { CLG_FERMION_WILSON = 0, CLG_FERMION_STAGGERED = 1 } clg_fermion_kind;
typedef enum { CLG_SUBSET_FULL = 0, CLG_SUBSET_EVEN = 1 } clg_subset;
typedef enum { CLG_PREC_DOUBLE = 0, CLG_PREC_SINGLE = 1, CLG_PREC_HALF = 2 } clg_precision;
typedef enum { CLG_LAYOUT_CLGBIN = 0, CLG_LAYOUT_BRIDGEPP = 1 } clg_layout;
/* ZERO: all links 0 (a force accumulator, CFieldGaugeSU3::InitialField(EFIT_Zero)) */
typedef enum { CLG_GAUGE_IDENTITY = 0, CLG_GAUGE_HAAR = 1, CLG_GAUGE_EXPH = 2, CLG_GAUGE_ZERO = 3 } clg_gauge_init;
/* EFieldFileType (Data/Field/CField.h): CLGBin double / float (18 reals per
 * link, CLGBin order), CLGBin compressed (9 reals per link: log U; the
 * reference writes its build's Real, so both widths exist), Bridge++ binary
 * (big-endian doubles) and text (one value per line), Bridge++ site order */
typedef enum {
    CLG_FILE_CLGBIN_DOUBLE = 0,           /* EFFT_CLGBinDouble (EFFT_CLGBin in a double build)    */
    CLG_FILE_CLGBIN_FLOAT = 1,            /* EFFT_CLGBinFloat                                     */
    CLG_FILE_CLGBIN_COMPRESSED = 2,       /* EFFT_CLGBinCompressed, double build                  */
    CLG_FILE_CLGBIN_COMPRESSED_FLOAT = 3, /* EFFT_CLGBinCompressed, single-precision build        */
    CLG_FILE_BRIDGEPP_BIN = 4,            /* EFFT_BridgePPBin                                     */
    CLG_FILE_BRIDGEPP_TXT = 5             /* EFFT_BridgePPTXT                                     */
} clg_file_format;
/* Z2: (+-1 +- i)/sqrt 2 per component; Z4: one of 1, i, -1, -i per component
 * (EFIT_RandomZ4, Random.h _deviceRandomZ4) */
typedef enum { CLG_SOURCE_ZERO = 0, CLG_SOURCE_GAUSS = 1, CLG_SOURCE_Z2 = 2, CLG_SOURCE_POINT = 3, CLG_SOURCE_Z4 = 4 } clg_source_kind;
typedef enum {
    CLG_SOLVER_GMRES = 0,       /* CSLASolverGMRES    SparseLinearAlgebra/CSolverGMRES.cpp:111-358   */
    CLG_SOLVER_BICGSTAB = 1,    /* CSLASolverBiCGStab SparseLinearAlgebra/CSolverBiCGstab.cpp:403-607 */
    CLG_SOLVER_CG = 2,          /* CG on Hermitian positive operators (DD^+, staggered (DD^+)_ee)     */
    CLG_SOLVER_CGM = 3,         /* multi-shift CG (no reference twin; CMultiShiftSolver.h:38-47 API)  */
    CLG_SOLVER_FOM_MS = 4,      /* CMultiShiftFOM     SparseLinearAlgebra/CMultiShiftFOM.cpp:97-270   */
    CLG_SOLVER_GCRODR = 5,      /* CSLASolverGCRODR   SparseLinearAlgebra/CSolverGCRODR.cpp:196-911   */
    CLG_SOLVER_NESTED_MS = 6,   /* CMultiShiftNested  SparseLinearAlgebra/CMultiShiftNested.cpp:69-145 */
    CLG_SOLVER_BICGSTAB_MS = 7, /* CMultiShiftBiCGStab SparseLinearAlgebra/CMultiShiftBiCGStab.cpp:73-437 */
    CLG_SOLVER_GMRESMDR = 8,    /* CSLASolverGMRESMDR SparseLinearAlgebra/CSolverGMRESMDR.cpp:16-170  */
    CLG_SOLVER_GMRES_MS = 9     /* CMultiShiftGMRES   SparseLinearAlgebra/CMultiShiftGMRES.cpp:113-330 */
} clg_solver_kind;

/* GCRO-DR deflation space (EEigenDeflationType, CSolverGCRODR.cpp:541-760):
 * SVD the k smallest eigenpairs of G^+ G p = l diag(U^+ U, 1) p (the reference's default),
 * REV the k smallest Ritz pairs W^+ A W p = l W^+ W p,
 * HEV the k largest of G^+ What^+ W p = l G^+ G p (harmonic),
 * where A W = What G is the cycle's Arnoldi relation. */
typedef enum { CLG_DEFLATION_SVD = 0, CLG_DEFLATION_REV = 1, CLG_DEFLATION_HEV = 2 } clg_deflation;

/* ------------------------------------------------------------------ handles */
typedef struct clg_context_s* clg_context;
typedef struct clg_lattice_s* clg_lattice;
typedef struct clg_gauge_s* clg_gauge;
typedef struct clg_field_s* clg_field;
typedef struct clg_solver_s* clg_solver;

/* ------------------------------------------------------------------ context
 * Replaces appInitialCLG / CCLGLibManager::InitialWithParameter device setup
 * (Core/CLGLibManager.cpp:882-917).  stream == NULL creates a private stream.
 * Objects made on a context (lattices, gauge and fermion fields, solvers,
 * whose workspaces hold fields) are destroyed before the context. */
clg_status clg_context_create(int device, void* cuda_stream, clg_context* out);
clg_status clg_context_destroy(clg_context ctx);
clg_status clg_context_set_stream(clg_context ctx, void* cuda_stream);
clg_status clg_context_synchronize(clg_context ctx);
const char* clg_status_string(clg_status s);
const char* clg_last_error(clg_context ctx);
/* number of kernels this context has launched (all kinds), for accounting */
clg_status clg_context_kernel_count(clg_context ctx, int64_t* count);
/* the autotuner's choices so far, one "<kernel key>=<config>" per line (config
 * = block size | variant << 16); writes at most len bytes including the
 * terminating zero and stores the full length (without it) in *needed.  No
 * reference counterpart: the reference launches with fixed block sizes
 * (Core/CudaHelper.cu). */
clg_status clg_context_tuned(clg_context ctx, char* buf, size_t len, size_t* needed);

/* ------------------------------------------------------------------ lattice
 * Replaces InitialLatticeAndConstant (Core/CLGLibManager.cpp:52-348) and the
 * torus boundary tables (Data/Boundary/CBoundaryConditionTorusSquare.cu:18-64):
 * dims = (Lx,Ly,Lz,Lt), all even; fermion_bc = boundary sign per direction
 * (the reference default is (1,1,1,-1), Core/CLGLibManager.cpp:549-566). */
clg_status clg_lattice_create(clg_context ctx, const int dims[4], const int fermion_bc[4], clg_lattice* out);
clg_status clg_lattice_destroy(clg_lattice lat);

/* ------------------------------------------------------------------ gauge
 * CFieldGaugeSU3 (Data/Field/Gauge/CFieldGaugeSU3.h:18-121).
 * import: InitialFieldWithFile / InitialWithByte (CFieldGaugeSU3.cu:1080-1222),
 *   layout CLGBIN (EFFT_CLGBinDouble) or BRIDGEPP (_kernelSetConfigurationSU3,
 *   CFieldGaugeSU3.cu:568-592); `data` holds 4*V*18 doubles, on the host unless
 *   on_device != 0.
 * export: CopyDataOutDouble (CFieldGaugeSU3.cu:1693-1760), CLGBin order.
 * random: seeded Haar SU(3), exp(i eps H), identity or zero links generated on the device. */
clg_status clg_gauge_create(clg_lattice lat, clg_gauge* out);
clg_status clg_gauge_destroy(clg_gauge g);
clg_status clg_gauge_import(clg_gauge g, const double* data, int layout, int on_device);
clg_status clg_gauge_export(clg_gauge g, double* data, int on_device);
clg_status clg_gauge_random(clg_gauge g, int init, uint64_t seed, uint32_t field_id, double eps);
/* Files.  load: CFieldGaugeSU3::InitialFieldWithFile (CFieldGaugeSU3.cu:1080-1265),
 * every clg_file_format; the file size must match the lattice.  save:
 * CField::SaveToFile / SaveToCompressedFile (Data/Field/CField.cpp:32-72,
 * CFieldGaugeSU3.cu:1651-1690), md5_hex_out (nullable, 33 chars) receives the
 * MD5 of the bytes written as the reference returns it.  The reference writes
 * no Bridge++ files; here both Bridge++ forms can be written too.  Compressed
 * saves need SU(3) links (clg_gauge_unitarity < 1e-12). */
clg_status clg_gauge_load(clg_gauge g, const char* path, int format);
clg_status clg_gauge_save(clg_gauge g, const char* path, int format, char* md5_hex_out);
/* MD5 (RFC 1321) of a host buffer as 32 lowercase hex digits + NUL (CLGMD5Hash) */
clg_status clg_md5(const void* data, size_t bytes, char* md5_hex_out);
/* average (1/3) Re tr of the plaquette (TestConfigurationFileIO.cpp:12-38 known answer) */
clg_status clg_gauge_plaquette(clg_gauge g, double* out);
/* max |U U^+ - 1| and |det U - 1| over links; the 12-real FP32/FP16 copies are
 * built only when this is below 1e-12 */
clg_status clg_gauge_unitarity(clg_gauge g, double* out);

/* ------------------------------------------------------------------ fermion fields
 * CFieldFermionWilsonSquareSU3 (param = Hopping kappa, CFieldFermionWilsonSquareSU3.cu:637-654)
 * CFieldFermionKSSU3 (param = Mass = 2am, Data/Field/CField.cpp:150-195).
 * A field holds nrhs right-hand sides.  import/export move CLGBin-ordered
 * full-lattice data (V*24 or V*6 doubles per rhs); EVEN fields read / write
 * only the even sites of that array (odd sites are exported as zero). */
clg_status clg_field_create(clg_lattice lat, int kind, int subset, int precision, int nrhs, double param,
                            clg_field* out);
clg_status clg_field_destroy(clg_field f);
clg_status clg_field_set_param(clg_field f, double param);
clg_status clg_field_import(clg_field f, int rhs, const double* data, int on_device);
clg_status clg_field_export(clg_field f, int rhs, double* data, int on_device);
/* Asynchronous host transfers (no reference counterpart: the reference copies
 * synchronously, CFieldFermionWilsonSquareSU3.cu InitialFieldWithFile /
 * CopyDataOut).  They let a caller overlap the PCIe copies of one solve's
 * source and solution with the next solve; `data` should be pinned host memory.
 *
 * clg_field_import_async: the host-to-device copy starts at once on the
 * context's copy stream; the field takes the data before the next operation
 * that uses it (any call taking the field), which waits for the copy.  `data`
 * must stay unchanged until clg_field_wait(f) returns.
 *
 * clg_field_export_async: queued on the context stream after the work issued
 * so far (the field's current value), copied to `data` on the copy stream;
 * `data` is complete once clg_field_wait(f) returns.
 *
 * clg_field_wait: waits for every asynchronous transfer of f issued so far. */
clg_status clg_field_import_async(clg_field f, int rhs, const double* data);
clg_status clg_field_export_async(clg_field f, int rhs, double* data);
clg_status clg_field_wait(clg_field f);
/* InitialField / InitialAsSource (CFieldFermionWilsonSquareSU3.cu:1102-1136, :521-566):
 * GAUSS (E|z|^2 = 1), Z2 ((+-1 +- i)/sqrt 2), POINT (site, spin*3+colour), ZERO. */
clg_status clg_field_random(clg_field f, int rhs, int kind, uint64_t seed, uint32_t field_id, int64_t site, int comp);
clg_status clg_field_copy(clg_field dst, clg_field src);  /* CopyTo; converts precision */
/* CField::SaveToFile / InitialFieldWithFile for fermion fields: one right-hand
 * side as CLGBin double or float (24 or 6 reals per site, CLGBin order) */
clg_status clg_field_save(clg_field f, int rhs, const char* path, int format, char* md5_hex_out);
clg_status clg_field_load(clg_field f, int rhs, const char* path, int format);

/* ------------------------------------------------------------------ operators
 * CField::ApplyOperator (Data/Field/CField.h:203): in place, the field is both
 * input and output; coefficient EOCT_None / Minus / Real / Complex. */
clg_status clg_apply(int op, clg_field inout, clg_gauge g, int coeff_type, double cre, double cim);
/* out-of-place variant: out = coeff * op(in) */
clg_status clg_apply_to(int op, clg_field out, clg_field in, clg_gauge g, int coeff_type, double cre, double cim);

/* ------------------------------------------------------------------ BLAS
 * CField BLAS (Data/Field/CField.h:127-201): Dot = sum conj(a) b, accumulated in
 * FP64 (re_im holds 2*nrhs doubles), Axpy, ScalarMultply, Zero, CopyTo. */
clg_status clg_dot(clg_field a, clg_field b, double* re_im);
/* No counterpart in the reference.  clg_dot without any device allocation, for
 * callers that may not call cudaMalloc: code that gives all device memory to its
 * own pool up front, code under a fixed device-memory budget, or a hot loop that
 * cannot afford the device-wide synchronisation cudaMalloc / cudaFree imply.
 * Same result as clg_dot; the scratch lives in one fixed 64 KiB __device__
 * array of the library (held on every GPU that loads it until exit), so at most
 * CLG_DOT_NOALLOC_MAX_RHS right-hand sides (CLG_ERR_BAD_ARG beyond).
 * clg_context_create looks the array up and loads its kernels on the context's
 * device (the point where lazy module loading gives them device memory), so no
 * call of this entry point allocates; create the context before handing the
 * rest of the GPU to another pool.  All calls share the array: calls that
 * overlap on one GPU race. */
#define CLG_DOT_NOALLOC_MAX_RHS 64
clg_status clg_dot_noalloc(clg_field a, clg_field b, double* re_im);
clg_status clg_norm2(clg_field a, double* out);
clg_status clg_axpy(clg_field y, double are, double aim, clg_field x);
clg_status clg_scale(clg_field y, double are, double aim);
clg_status clg_zero(clg_field y);

/* ------------------------------------------------------------------ solvers
 * CSLASolver::Configurate keys (CSolverGMRES.cpp:35-99, CSolverBiCGstab.cpp:33-93)
 * plus the B200 options.  tol_true_rel is the true relative residual
 * |b - M x| / |b| every solve must reach, recomputed in FP64. */
typedef struct {
    int32_t kind;              /* clg_solver_kind                                         */
    int32_t max_dim;           /* MaxDim (GMRES / FOM Krylov dimension)                   */
    int32_t restart;           /* Restart (cycles)                                        */
    double accuracy;           /* Accuracy (reference stopping quantity, squared)          */
    int32_t absolute_accuracy; /* AbsoluteAccuracy                                        */
    int32_t deviation_step;    /* DiviationStep (BiCGStab)                                */
    int32_t max_step;          /* MaxStep (BiCGStab)                                      */
    double small_rho;          /* SmallRho (BiCGStab)                                     */
    int32_t inner_precision;   /* clg_precision of the Krylov iterations                  */
    double tol_true_rel;       /* required true relative residual (FP64), e.g. 1e-10     */
    double inner_tol;          /* relative reduction per defect-correction cycle          */
    int32_t max_iterations;    /* total operator applications allowed                     */
    int32_t max_outer;         /* defect-correction cycles allowed                        */
    int32_t even_odd;          /* solve D x = b through the even-odd Schur system         */
    int32_t use_graphs;        /* capture the inner iterations in CUDA graphs             */
    int32_t kdim;              /* KDim (GCRO-DR recycled dimension; 0: MaxDim - 2)         */
    int32_t deflation;         /* DeflateSpace (GCRO-DR): clg_deflation, default SVD      */
} clg_solver_params;

typedef struct {
    int32_t status;            /* clg_status of this right-hand side / shift              */
    int32_t iterations;        /* operator applications (all precisions)                  */
    int32_t restarts;          /* restart cycles                                          */
    int32_t outer;             /* defect-correction cycles                                */
    double true_rel_residual;  /* |b - M x| / |b| in FP64 at exit                          */
    double seconds;            /* wall time of the call                                   */
} clg_solve_info;

clg_status clg_solver_default_params(int kind, clg_solver_params* p);
clg_status clg_solver_create(clg_context ctx, const clg_solver_params* p, clg_solver* out);
clg_status clg_solver_destroy(clg_solver s);
/* GCRO-DR keeps its recycled subspace U_k between clg_solve calls on the same
 * lattice and operator (the reference's ESP_InTrajectory phase); this drops it
 * (ESP_StartTrajectory).  No effect on the other solver kinds. */
clg_status clg_solver_reset(clg_solver s);
/* CSLASolver::Solve (SparseLinearAlgebra/CSLASolver.h:42-50): solve op x = b for
 * every right-hand side of b; x may alias b; x0 (nullable) is the start vector
 * (pStart).  info holds nrhs entries.  Returns CLG_SUCCESS only when every
 * right-hand side reached tol_true_rel.
 * GCRO-DR (CLG_SOLVER_GCRODR): FP64 fields, one right-hand side, max_dim = MDim
 * (5..32), kdim = KDim (2..MDim-2), deflation = DeflateSpace, restart = cycles, x0 = b when no start
 * vector is given (CSolverGCRODR.cpp:216-223); inner_precision is not used.
 * GMRES-MDR (CLG_SOLVER_GMRESMDR): the same parameters and cycles; a solve that
 * starts from a kept U_k first rotates it to the eigenvectors of the deflation
 * type's k x k problem on span U_k (GenerateCUFirstTime, CSolverGMRESMDR.cpp:16-135),
 * with C_k = A U_k made orthonormal again (the reference leaves C_k = A Q). */
clg_status clg_solve(clg_solver s, clg_field x, clg_field b, clg_gauge g, int op, clg_field x0, clg_solve_info* info);
/* CMultiShiftSolver::Solve (SparseLinearAlgebra/CMultiShiftSolver.h:38-47):
 * (op + c_n) x_n = b for n < nshift; shifts_re_im holds nshift complex shifts
 * (real for CGM); x[n] must not alias b (CMultiShiftSolver.h:35).
 *   CLG_SOLVER_CGM: multi-shift CG over one Krylov space (Hermitian positive
 *     op, real shifts >= 0): the shared iteration in FP64 until |r| <= inner_tol
 *     |b| (default 1e-4), then in the inner precision, the shifted x_n, p_n in
 *     FP64; every shift's FP64 true residual is checked and, if needed, refined.
 *   CLG_SOLVER_FOM_MS: restarted FOM(max_dim <= 32) over one Krylov space for
 *     every complex shift, FP64 (b and x FP64), restart = cycles, stop when every
 *     shift's residual |beta_n| <= tol_true_rel |b|; then the true residuals are
 *     checked in FP64 and refined if needed.
 *   CLG_SOLVER_GMRES_MS: restarted GMRES(max_dim <= 32) on the unshifted seed
 *     system with every shift's residual kept collinear with the seed's
 *     (Frommer-Glaessner), FP64, restart = cycles; then checked and refined.
 *   CLG_SOLVER_BICGSTAB_MS: BiCGStab-M (shadow residual conj(b)) over one Krylov
 *     space for every complex shift, FP64, checked every deviation_step
 *     iterations, at most max_step * deviation_step iterations; then checked and
 *     refined like FOM_MS.
 *   CLG_SOLVER_NESTED_MS: every shift solved as one right-hand side of a batched
 *     shifted solve (GMRES / CG in the inner precision, FP64 defect correction):
 *     the batched form of CMultiShiftNested, no shared Krylov space. */
clg_status clg_solve_multishift(clg_solver s, clg_field* x, int nshift, const double* shifts_re_im, clg_field b,
                                clg_gauge g, int op, clg_solve_info* info);
/* Several lattices of uneven volume in one solve (no reference counterpart:
 * the reference holds one lattice per process, Core/CudaHelper.cu:14-25, and
 * changes it with appQuitCLG / appInitialCLG, Core/CLGLibManager.cpp:1131-1162).
 * Lattice i: x[i], b[i] FULL FP64 Wilson fields with the same nrhs and U[i] its
 * gauge field; one hopping parameter; op = CLG_OP_D or CLG_OP_DDAG; a GMRES,
 * BiCGStab or CG solver (CG: CGNE on the even-odd system), low-precision inner
 * solves need SU(3) links.  Every right-hand side of every lattice is one
 * right-hand side of a single solve (one kernel per step covers all lattices);
 * info holds sum_i nrhs_i entries in lattice order. */
clg_status clg_solve_lattices(clg_solver s, int n, clg_field* x, clg_field* b, clg_gauge* U, int op,
                              clg_solve_info* info);
/* CFieldFermion::RationalApproximation (Data/Field/CField.cpp:114-145):
 * f <- c f + sum_i a_i (op + b_i)^{-1} f through one multi-shift solve. */
clg_status clg_rational_apply(clg_solver s, clg_field f, clg_gauge g, int op, int degree, double c,
                              const double* a, const double* b, clg_solve_info* info);

/* Small dense eigenproblems of the recycled solver (host code, no device):
 * A x = w x (b == NULL) or A x = w B x with B Hermitian positive definite,
 * n <= 64, row-major interleaved complex; w receives n eigenvalues and the
 * columns of x (row-major n x n) the unit eigenvectors (the reference's
 * CLinearAlgebraHelper::EigenValueProblem / GeneralizedEigenValueProblem,
 * Tools/Math/CLinearAlgebraHelper.cu:2155-2610, which run on the device). */
clg_status clg_small_eig(int n, const double* a, const double* b, double* w, double* x);

/* ------------------------------------------------------------------ HMC fermion force
 * CFieldFermionWilsonSquareSU3::DerivateDOperator / _kernelDWilsonForceSU3
 * (Data/Field/WilsonDirac/CFieldFermionWilsonSquareSU3.cu:170-231, :260-275):
 * with X = (D D^+)^-1 phi and Y = D^+ X (FULL FP64 Wilson fields, kappa = X's
 * param), add to every link
 *   F_mu(x) += s kappa Ta(U_mu(x) [sum_s ((1 - g_mu) Y(x+mu))_s X(x)_s^+ + X(x+mu)_s ((1 + g_mu) Y(x))_s^+])
 * (Ta the traceless anti-hermitian part, s the fermion boundary sign of the hop
 * x -> x+mu).  F is a gauge field used as an accumulator (start it with
 * clg_gauge_random(F, CLG_GAUGE_ZERO, ...)); it must not be g.  Fields holding
 * several right-hand sides add the force of each. */
clg_status clg_wilson_force(clg_gauge F, clg_gauge g, clg_field X, clg_field Y);
/* CFieldFermionWilsonSquareSU3::CalculateForceS (same file :1016-1100): solve
 * D D^+ X = phi with solver s (start vector `cache` when given, the reference's
 * CachedInverseDDdaggerField), store X in `cache`, Y = D^+ X, then
 * clg_wilson_force(F, g, X, Y).  X and Y are kept by the solver between calls.
 * A solve that fails returns its status and adds nothing to F. */
clg_status clg_wilson_fermion_force(clg_solver s, clg_gauge F, clg_gauge g, clg_field phi, clg_field cache,
                                    clg_solve_info* info);
/* CFieldFermionKSSU3::DerivateD0 / _kernelDFermionKSForce
 * (Data/Field/Staggered/CFieldFermionKSSU3.cu:216-262, :316-331): with the
 * multi-shift solutions phi_i[i] = (D D^+ + b_i)^-1 phi and phi_id[i] = D0 phi_i[i]
 * (massless D; FULL FP64 staggered fields of one right-hand side), n <= 64
 * poles with numerators a[i], subtract from every link
 *   F_mu(x) -= sum_i Ta(s eta_mu(x) a_i [U_mu(x) phi_i(x+mu) phi_id(x)^+ + phi_i(x) (U_mu(x) phi_id(x+mu))^+])
 * (s the fermion boundary sign of the hop x -> x+mu, eta_mu the staggered phase). */
clg_status clg_ks_force(clg_gauge F, clg_gauge g, int n, const clg_field* phi_i, const clg_field* phi_id,
                        const double* a);
/* CFieldFermionKSSU3::CalculateForceS (same file :412-500): one multi-shift
 * solve (s is a CGM or FOM_MS solver) of (D D^+ + b_i) phi_i = phi for the
 * `degree` poles of the molecular-dynamics rational approximation (numerators
 * a, shifts b: the reference's m_rMD), phi_id = D0 phi_i, then clg_ks_force.
 * info holds `degree` entries.  A failed solve adds nothing to F. */
clg_status clg_ks_fermion_force(clg_solver s, clg_gauge F, clg_gauge g, clg_field phi, int degree, const double* a,
                                const double* b, clg_solve_info* info);

/* ------------------------------------------------------------------ measurements
 * EGammaMatrix (Core/CudaHelper.h:37-63), chiral set and products as
 * gammaMatrixSet::CreateGammaMatrix (Tools/Math/GammaMatrix.h:405-511). */
typedef enum {
    CLG_GAMMA_UNITY = 0, CLG_GAMMA1, CLG_GAMMA2, CLG_GAMMA3, CLG_GAMMA4, CLG_GAMMA5, CLG_GAMMA51, CLG_GAMMA52,
    CLG_GAMMA53, CLG_GAMMA54, CLG_GAMMA15, CLG_GAMMA25, CLG_GAMMA35, CLG_GAMMA45, CLG_SIGMA12, CLG_SIGMA23,
    CLG_SIGMA31, CLG_SIGMA41, CLG_SIGMA42, CLG_SIGMA43, CLG_SIGMA12E, CLG_SIGMA23E, CLG_SIGMA31E, CLG_CHARGECONJG,
    CLG_GAMMA_COUNT
} clg_gamma;
/* CMeasureMesonCorrelator::CalculateCorrelator (Measurement/CMeasureMesonCorrelator.cu:254-411):
 * the 12 spin-colour point sources at the origin solved in one batched call of
 * solver s into prop (a FULL FP64 Wilson field of 12 right-hand sides, rhs =
 * spin*3 + colour, kappa = its param; info holds 12 entries), then
 * clg_meson_contract.  corr receives ngamma x Lt doubles, corr[k*Lt + t]. */
clg_status clg_meson_correlator(clg_solver s, clg_gauge g, clg_field prop, int ngamma, const int* gammas, double* corr,
                                clg_solve_info* info);
/* _kernelCalculateCorrelatorSU3 (same file :26-174) on given propagators and the
 * spatial sums per time slice times 2/sqrt(V) (:366-380) */
clg_status clg_meson_contract(clg_field prop, int ngamma, const int* gammas, double* corr);
/* Stochastic condensate (CMeasurementManager.cpp:71-115 with
 * CMeasureChiralCondensate::OnConfigurationAcceptedZ4SingleField,
 * Measurement/CMeasureChiralCondensate.cu:236-290): one Z4 noise vector per
 * right-hand side of eta (seed, field id = rhs + 1), psi = D^-1 eta in one
 * batched solve, then the nine traces of clg_condensate_contract averaged over
 * the noise vectors: re_im receives 9 complex numbers. */
clg_status clg_chiral_condensate(clg_solver s, clg_gauge g, clg_field eta, clg_field psi, uint64_t seed, double* re_im,
                                 clg_solve_info* info);
/* _kernelDotMeasureAll (same file :38-100) summed over sites: per right-hand
 * side r and kind k, (1/V) sum_x eta_r(x)^+ Gamma_k psi_r(x) into
 * re_im[(r*9 + k)*2 + {0, 1}], Gamma_k = 1, gamma1..gamma5, gamma4 gamma5,
 * gamma1, gamma2 (the last two are the reference's rotating-frame kinds 7 and 8
 * at omega = 0) */
clg_status clg_condensate_contract(clg_field eta, clg_field psi, double* re_im);

#ifdef __cplusplus
}
#endif
#endif
