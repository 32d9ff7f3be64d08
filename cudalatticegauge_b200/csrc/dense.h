// dense.h -- small dense complex linear algebra on the host for the recycled
// Krylov solver (matrices of order <= 33): thin QR, least squares, the complex
// Schur form and eigenvectors of a general matrix, and the generalized
// problem A p = l B p with B Hermitian positive definite.
//
// Methods (Golub & Van Loan, Matrix Computations, 4th ed.): classical
// Gram-Schmidt with one reorthogonalisation for QR (5.2.8); Householder
// reduction to Hessenberg form (7.4.3) and the implicitly shifted complex QR
// iteration with Wilkinson shifts and Givens bulge chasing to the Schur form
// (7.5); eigenvectors by back substitution on the triangular factor (7.6.4).
// A p = l B p is reduced to R^-1 Q^+ A with B = QR.
#pragma once
#include <complex>
#include <vector>

namespace clg {
namespace dense {

using Z = std::complex<double>;

// row-major rows x cols
struct Mat {
  int rows = 0, cols = 0;
  std::vector<Z> a;
  Mat() {}
  Mat(int r, int c) : rows(r), cols(c), a((size_t)r * c, Z(0.0, 0.0)) {}
  Z& operator()(int i, int j) { return a[(size_t)i * cols + j]; }
  const Z& operator()(int i, int j) const { return a[(size_t)i * cols + j]; }
};

Mat mul(const Mat& A, const Mat& B);            // A B
Mat mul_dag(const Mat& A, const Mat& B);        // A^+ B
// thin QR of an n x k matrix (n >= k): Q n x k with orthonormal columns, R k x k upper triangular
bool qr_thin(const Mat& A, Mat& Q, Mat& R);
// argmin_y |c - G y| for G n x m (n >= m, full column rank)
bool lstsq(const Mat& G, const std::vector<Z>& c, std::vector<Z>& y);
// eigenvalues / unit eigenvectors (columns of X) of a general square matrix;
// false when the QR iteration does not converge
bool eig(const Mat& A, std::vector<Z>& w, Mat& X);
// A p = l B p, B Hermitian positive definite
bool geig(const Mat& A, const Mat& B, std::vector<Z>& w, Mat& X);
// the k eigenvectors (as the columns of an n x k matrix) whose eigenvalues have
// the smallest (smallest = true) or largest modulus
Mat select(const std::vector<Z>& w, const Mat& X, int k, bool smallest);

}  // namespace dense
}  // namespace clg
