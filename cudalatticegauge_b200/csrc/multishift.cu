// multishift.cu -- CMultiShiftSolver::Solve (SparseLinearAlgebra/CMultiShiftSolver.h:38-47)
// and CFieldFermion::RationalApproximation (Data/Field/CField.cpp:114-145).
#include "internal.h"

extern "C" {

clg_status clg_solve_multishift(clg_solver s, clg_field* x, int nshift, const double* shifts, clg_field b, clg_gauge g,
                                int op, clg_solve_info* info) {
  (void)x; (void)nshift; (void)shifts; (void)b; (void)g; (void)op; (void)info;
  if (!s) return CLG_ERR_BAD_ARG;
  return CLG_ERR_UNSUPPORTED;
}

clg_status clg_rational_apply(clg_solver s, clg_field f, clg_gauge g, int op, int degree, double c, const double* a,
                              const double* b, clg_solve_info* info) {
  (void)f; (void)g; (void)op; (void)degree; (void)c; (void)a; (void)b; (void)info;
  if (!s) return CLG_ERR_BAD_ARG;
  return CLG_ERR_UNSUPPORTED;
}

}  // extern "C"
