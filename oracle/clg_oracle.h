/*
 * clg_oracle.h -- FP64 CPU restatement of CLGLib's fermion hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it; the product
 * library (libclgb200.so) never links it and never falls back to it.
 *
 * Every function states the reference file:line whose behaviour it restates
 * (paths relative to the CudaLatticeGauge source tree).  Conventions:
 *
 *  - site index  s = ((x*Ly + y)*Lz + z)*Lt + t            (Data/CCommonData.h:274-277)
 *  - link index  l = s*4 + mu, mu = 0..3 = x,y,z,t           (Data/CCommonData.h:324-327)
 *  - gauge link: 9 complex, row-major, (re,im) interleaved  (CFieldGaugeSU3.cu:1199-1222, CLGBin order)
 *  - Wilson spinor: 4 spins x 3 colours complex, spin-major (Tools/Math/Vectors.h:575-888)
 *  - staggered vector: 3 colours complex                    (Tools/Math/Vectors.h:287-571)
 *  - fermion boundary sign per direction bc[mu] = +1/-1      (CBoundaryConditionTorusSquare.cu:18-64;
 *    default (1,1,1,-1), Core/CLGLibManager.cpp:549-566); gauge links are periodic.
 *
 * All arrays are interleaved (re,im) doubles.  Lengths are given in complex numbers.
 */
#ifndef CLG_ORACLE_H
#define CLG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int L[4];   /* Lx, Ly, Lz, Lt */
    int bc[4];  /* fermion boundary sign per direction (+1 periodic, -1 antiperiodic) */
} clgo_lat;

/* ---------------------------------------------------------------- RNG / fields */
void clgo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void clgo_gen_gauge_haar(const int L[4], uint64_t seed, uint32_t field_id, double* U);
void clgo_gen_gauge_expH(const int L[4], uint64_t seed, uint32_t field_id, double eps, double* U);
void clgo_gen_gauge_identity(const int L[4], double* U);
void clgo_gen_gauss(long nsites, int ncomp, uint64_t seed, uint32_t field_id, double* psi);
void clgo_gen_z2(long nsites, int ncomp, uint64_t seed, uint32_t field_id, double* psi);
void clgo_gen_z4(long nsites, int ncomp, uint64_t seed, uint32_t field_id, double* psi);
void clgo_gen_point(long nsites, int ncomp, long site, int comp, double* psi);
void clgo_zero_parity(const int L[4], int ncomp, int parity, double* psi);
double clgo_plaquette(const int L[4], const double* U);
double clgo_unitarity_deviation(long nlinks, const double* U);
void clgo_bridgepp_to_clg(const int L[4], const double* bridge, double* U);

/* ---------------------------------------------------------------- operators  */
/* coefficient types: EOCT_None / Minus / Real / Complex (Data/Field/CField.h:62-68) */
enum { CLGO_EOCT_NONE = 0, CLGO_EOCT_MINUS = 1, CLGO_EOCT_REAL = 2, CLGO_EOCT_COMPLEX = 3 };

void clgo_wilson_D(const clgo_lat* lat, const double* U, double kappa, int dagger,
                   int coeff_type, double cre, double cim, const double* in, double* out);
void clgo_wilson_hop(const clgo_lat* lat, const double* U, int dagger, int out_parity,
                     const double* in, double* out);
void clgo_wilson_mee(const clgo_lat* lat, const double* U, double kappa, int dagger,
                     const double* in, double* out, double* tmp);
/* F += Wilson fermion force from X = (DD^+)^-1 phi and Y = D^+ X (link layout of U) */
void clgo_wilson_force(const clgo_lat* lat, const double* U, double kappa, const double* X, const double* Y,
                       double* F);
void clgo_ks_D(const clgo_lat* lat, const double* U, double mass2am, int dagger,
               int coeff_type, double cre, double cim, const double* in, double* out);
void clgo_ks_hop(const clgo_lat* lat, const double* U, int out_parity, const double* in, double* out);
/* F -= staggered rational force of phi_i = (DD^+ + b_i)^-1 phi, phi_id = D0 phi_i, numerators a (n fields each) */
void clgo_ks_force(const clgo_lat* lat, const double* U, int n, const double* phi_i, const double* phi_id,
                   const double* a, double* F);
void clgo_ks_dddag_ee(const clgo_lat* lat, const double* U, double mass2am,
                      const double* in, double* out, double* tmp);

/* ---------------------------------------------------------------- measurements */
/* EGammaMatrix (Core/CudaHelper.h:37-63) */
enum {
    CLGO_UNITY = 0, CLGO_GAMMA1, CLGO_GAMMA2, CLGO_GAMMA3, CLGO_GAMMA4, CLGO_GAMMA5, CLGO_GAMMA51, CLGO_GAMMA52,
    CLGO_GAMMA53, CLGO_GAMMA54, CLGO_GAMMA15, CLGO_GAMMA25, CLGO_GAMMA35, CLGO_GAMMA45, CLGO_SIGMA12, CLGO_SIGMA23,
    CLGO_SIGMA31, CLGO_SIGMA41, CLGO_SIGMA42, CLGO_SIGMA43, CLGO_SIGMA12E, CLGO_SIGMA23E, CLGO_SIGMA31E,
    CLGO_CHARGECONJG, CLGO_EGM_MAX
};
/* chiral gamma matrix `which`: row r -> column idx[r] with phase i^z[r]; next symmetric index */
int clgo_gamma(int which, int idx[4], int z[4], int* next_symmetric);
/* meson correlator C(t), t < Lt, of 12 propagators prop[r = spin*3 + colour] (each V*12 complex) */
void clgo_meson_correlator(const int L[4], const double* prop, int gamma, double* C);
/* (1/V) sum_x eta(x)^+ Gamma_kind psi(x), kind 0..8 as _kernelDotMeasureAll at omega = 0 */
void clgo_condensate(long V, const double* eta, const double* psi, int kind, double* re_im);

/* generic operator descriptor used by the solvers */
enum {
    CLGO_OP_WILSON_D = 0, CLGO_OP_WILSON_DDAG = 1, CLGO_OP_WILSON_DDDAG = 2, CLGO_OP_WILSON_DD = 3,
    CLGO_OP_WILSON_MEE = 4, CLGO_OP_WILSON_MEE_DAG = 5, CLGO_OP_WILSON_MEE_MEEDAG = 6,
    CLGO_OP_KS_D = 10, CLGO_OP_KS_DDAG = 11, CLGO_OP_KS_DDDAG = 12, CLGO_OP_KS_DDDAG_EE = 13
};
typedef struct {
    int kind;
    clgo_lat lat;
    const double* U;
    double param;     /* kappa (Wilson) or 2am (staggered) */
    double* tmp;      /* scratch, one field */
    double* tmp2;     /* scratch, one field */
} clgo_op;
long clgo_op_len(const clgo_op* op);
void clgo_apply(const clgo_op* op, const double* in, double* out);

/* ---------------------------------------------------------------- BLAS      */
void clgo_dot(long n, const double* a, const double* b, double* re_im);   /* sum conj(a) b */
double clgo_norm2(long n, const double* a);
void clgo_axpy(long n, double are, double aim, const double* x, double* y); /* y += a x   */

/* ---------------------------------------------------------------- solvers   */
typedef struct {
    int iterations;      /* operator applications */
    int restarts;
    int converged;
    double last_deviation;  /* the reference's stopping quantity at exit */
    double true_rel_residual;
} clgo_info;

int clgo_gmres(const clgo_op* op, const double* b, double* x, const double* x0,
               int maxdim, int restart, double accuracy, int absolute, clgo_info* info);
int clgo_bicgstab(const clgo_op* op, const double* b, double* x, const double* x0,
                  int dev_step, int max_step, int restart, double accuracy, int absolute,
                  double small_rho, int std_omega, clgo_info* info);
int clgo_cg(const clgo_op* op, const double* b, double* x, double tol_rel, int maxiter, clgo_info* info);
int clgo_cgm(const clgo_op* op, const double* b, int nshift, const double* shifts, double* x,
             double tol_rel, int maxiter, clgo_info* info);
int clgo_fom_ms(const clgo_op* op, const double* b, int nshift, const double* shifts_c, double* x,
                int maxdim, int restart, double accuracy, int absolute, clgo_info* info);
int clgo_bicgstab_ms(const clgo_op* op, const double* b, int nshift, const double* shifts_c, double* x,
                     int dev_step, int max_step, double accuracy, int absolute, clgo_info* info);
int clgo_gmres_ms(const clgo_op* op, const double* b, int nshift, const double* shifts_c, double* x,
                  int maxdim, int restart, double accuracy, int absolute, clgo_info* info);
double clgo_true_residual(const clgo_op* op, const double* b, const double* x, double shift_re, double shift_im);

#ifdef __cplusplus
}
#endif
#endif
