// dense.cu -- host implementation of dense.h (see there for the methods).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "dense.h"
#include "../../include/clg_b200.h"

namespace clg {
namespace dense {

namespace {
constexpr double EPS = 2.220446049250313e-16;

double fro(const Mat& A) {
  double s = 0.0;
  for (const Z& z : A.a) s += std::norm(z);
  return std::sqrt(s);
}
}  // namespace

Mat mul(const Mat& A, const Mat& B) {
  Mat C(A.rows, B.cols);
  for (int i = 0; i < A.rows; ++i)
    for (int l = 0; l < A.cols; ++l) {
      const Z a = A(i, l);
      if (a == Z(0.0, 0.0)) continue;
      for (int j = 0; j < B.cols; ++j) C(i, j) += a * B(l, j);
    }
  return C;
}

Mat mul_dag(const Mat& A, const Mat& B) {
  Mat C(A.cols, B.cols);
  for (int l = 0; l < A.rows; ++l)
    for (int i = 0; i < A.cols; ++i) {
      const Z a = std::conj(A(l, i));
      if (a == Z(0.0, 0.0)) continue;
      for (int j = 0; j < B.cols; ++j) C(i, j) += a * B(l, j);
    }
  return C;
}

bool qr_thin(const Mat& A, Mat& Q, Mat& R) {
  const int n = A.rows, k = A.cols;
  Q = Mat(n, k);
  R = Mat(k, k);
  const double scale = fro(A);
  for (int j = 0; j < k; ++j) {
    std::vector<Z> v(n);
    for (int i = 0; i < n; ++i) v[i] = A(i, j);
    for (int pass = 0; pass < 2; ++pass)
      for (int l = 0; l < j; ++l) {
        Z d(0.0, 0.0);
        for (int i = 0; i < n; ++i) d += std::conj(Q(i, l)) * v[i];
        R(l, j) += d;
        for (int i = 0; i < n; ++i) v[i] -= d * Q(i, l);
      }
    double nv = 0.0;
    for (int i = 0; i < n; ++i) nv += std::norm(v[i]);
    nv = std::sqrt(nv);
    if (!(nv > 1e-14 * scale) || !(nv > 1e-300)) return false;  // (numerically) rank deficient
    R(j, j) = nv;
    for (int i = 0; i < n; ++i) Q(i, j) = v[i] / nv;
  }
  return true;
}

bool lstsq(const Mat& G, const std::vector<Z>& c, std::vector<Z>& y) {
  Mat Q, R;
  if (!qr_thin(G, Q, R)) return false;
  const int m = G.cols;
  std::vector<Z> q(m, Z(0.0, 0.0));
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < G.rows; ++i) q[j] += std::conj(Q(i, j)) * c[i];
  y.assign(m, Z(0.0, 0.0));
  for (int j = m - 1; j >= 0; --j) {
    Z s = q[j];
    for (int l = j + 1; l < m; ++l) s -= R(j, l) * y[l];
    y[j] = s / R(j, j);
  }
  return true;
}

bool eig(const Mat& A0, std::vector<Z>& w, Mat& X) {
  const int n = A0.rows;
  Mat H = A0, Q(n, n);
  for (int i = 0; i < n; ++i) Q(i, i) = 1.0;
  const double anorm = std::max(fro(A0), 1e-300);
  // Householder reduction to upper Hessenberg form, H = Q^+ A Q
  for (int j = 0; j + 2 < n; ++j) {
    double xn = 0.0;
    for (int i = j + 1; i < n; ++i) xn += std::norm(H(i, j));
    xn = std::sqrt(xn);
    if (xn < 1e-300) continue;
    const Z x0 = H(j + 1, j);
    const Z ph = std::abs(x0) > 0 ? x0 / std::abs(x0) : Z(1.0, 0.0);
    std::vector<Z> v(n, Z(0.0, 0.0));
    for (int i = j + 1; i < n; ++i) v[i] = H(i, j);
    v[j + 1] += ph * xn;  // v = x + e^{i arg x0} |x| e_1
    double vn = 0.0;
    for (int i = j + 1; i < n; ++i) vn += std::norm(v[i]);
    vn = std::sqrt(vn);
    for (int i = j + 1; i < n; ++i) v[i] /= vn;
    // H <- (I - 2 v v^+) H (I - 2 v v^+),  Q <- Q (I - 2 v v^+)
    for (int col = 0; col < n; ++col) {
      Z d(0.0, 0.0);
      for (int i = j + 1; i < n; ++i) d += std::conj(v[i]) * H(i, col);
      for (int i = j + 1; i < n; ++i) H(i, col) -= 2.0 * v[i] * d;
    }
    for (int row = 0; row < n; ++row) {
      Z d(0.0, 0.0);
      for (int i = j + 1; i < n; ++i) d += H(row, i) * v[i];
      for (int i = j + 1; i < n; ++i) H(row, i) -= 2.0 * d * std::conj(v[i]);
      Z e(0.0, 0.0);
      for (int i = j + 1; i < n; ++i) e += Q(row, i) * v[i];
      for (int i = j + 1; i < n; ++i) Q(row, i) -= 2.0 * e * std::conj(v[i]);
    }
    for (int i = j + 2; i < n; ++i) H(i, j) = 0.0;
  }
  // shifted QR iteration to the Schur form, H = Q^+ A Q upper triangular
  int hi = n - 1, iter = 0, total = 0;
  while (hi > 0) {
    int l = hi;
    for (; l > 0; --l) {
      double s = std::abs(H(l - 1, l - 1)) + std::abs(H(l, l));
      if (s == 0.0) s = anorm;
      if (std::abs(H(l, l - 1)) < EPS * s) {
        H(l, l - 1) = 0.0;
        break;
      }
    }
    if (l == hi) {
      --hi;
      iter = 0;
      continue;
    }
    if (++total > 60 * n) return false;
    ++iter;
    Z mu;
    if (iter % 11 == 10) {
      mu = H(hi, hi) + std::abs(H(hi, hi - 1));  // exceptional shift
    } else {
      const Z a = H(hi - 1, hi - 1), b = H(hi - 1, hi), c = H(hi, hi - 1), d = H(hi, hi);
      const Z half = 0.5 * (a - d);
      const Z disc = std::sqrt(half * half + b * c);
      const Z m1 = 0.5 * (a + d) + disc, m2 = 0.5 * (a + d) - disc;
      mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
    }
    Z x = H(l, l) - mu, y = H(l + 1, l);
    for (int kk = l; kk < hi; ++kk) {
      // G = [[c, s], [-conj(s), c]] with G [x; y] = [r; 0]
      const double ax = std::abs(x), r = std::hypot(ax, std::abs(y));
      double c;
      Z s;
      if (r == 0.0) {
        c = 1.0;
        s = 0.0;
      } else if (ax == 0.0) {
        c = 0.0;
        s = 1.0;
      } else {
        c = ax / r;
        s = (x / ax) * std::conj(y) / r;
      }
      for (int col = (kk == l ? l : kk - 1); col < n; ++col) {
        const Z h1 = H(kk, col), h2 = H(kk + 1, col);
        H(kk, col) = c * h1 + s * h2;
        H(kk + 1, col) = -std::conj(s) * h1 + c * h2;
      }
      for (int row = 0; row <= std::min(kk + 2, hi); ++row) {
        const Z h1 = H(row, kk), h2 = H(row, kk + 1);
        H(row, kk) = h1 * c + h2 * std::conj(s);
        H(row, kk + 1) = -h1 * s + h2 * c;
      }
      for (int row = 0; row < n; ++row) {
        const Z q1 = Q(row, kk), q2 = Q(row, kk + 1);
        Q(row, kk) = q1 * c + q2 * std::conj(s);
        Q(row, kk + 1) = -q1 * s + q2 * c;
      }
      if (kk + 1 < hi) {
        x = H(kk + 1, kk);
        y = H(kk + 2, kk);
      }
    }
  }
  // eigenvectors of the triangular factor by back substitution, then X = Q Y
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = H(i, i);
  X = Mat(n, n);
  const double small = EPS * anorm;
  for (int i = 0; i < n; ++i) {
    std::vector<Z> yv(n, Z(0.0, 0.0));
    yv[i] = 1.0;
    for (int j = i - 1; j >= 0; --j) {
      Z s(0.0, 0.0);
      for (int l = j + 1; l <= i; ++l) s += H(j, l) * yv[l];
      Z den = H(j, j) - w[i];
      if (std::abs(den) < small) den = small;
      yv[j] = -s / den;
    }
    double nv = 0.0;
    std::vector<Z> xv(n, Z(0.0, 0.0));
    for (int r = 0; r < n; ++r) {
      for (int l = 0; l <= i; ++l) xv[r] += Q(r, l) * yv[l];
      nv += std::norm(xv[r]);
    }
    nv = std::sqrt(nv);
    for (int r = 0; r < n; ++r) X(r, i) = xv[r] / nv;
  }
  return true;
}

bool geig(const Mat& A, const Mat& B, std::vector<Z>& w, Mat& X) {
  const int n = A.rows;
  Mat Q, R;
  if (!qr_thin(B, Q, R)) return false;
  Mat M = mul_dag(Q, A);  // Q^+ A, then R^-1 (Q^+ A) column by column
  for (int j = 0; j < n; ++j)
    for (int i = n - 1; i >= 0; --i) {
      Z s = M(i, j);
      for (int l = i + 1; l < n; ++l) s -= R(i, l) * M(l, j);
      M(i, j) = s / R(i, i);
    }
  return eig(M, w, X);
}

Mat select(const std::vector<Z>& w, const Mat& X, int k, bool smallest) {
  const int n = (int)w.size();
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return smallest ? std::abs(w[a]) < std::abs(w[b]) : std::abs(w[a]) > std::abs(w[b]);
  });
  Mat P(X.rows, k);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < X.rows; ++i) P(i, j) = X(i, order[j]);
  return P;
}

}  // namespace dense
}  // namespace clg

using clg::dense::Mat;
using clg::dense::Z;

extern "C" {

clg_status clg_small_eig(int n, const double* a, const double* b, double* w, double* x) {
  if (n < 1 || n > 64 || !a || !w || !x) return CLG_ERR_BAD_ARG;
  Mat A(n, n), B(n, n);
  for (int i = 0; i < n * n; ++i) {
    A.a[i] = Z(a[2 * i], a[2 * i + 1]);
    if (b) B.a[i] = Z(b[2 * i], b[2 * i + 1]);
  }
  std::vector<Z> ev;
  Mat X;
  const bool ok = b ? clg::dense::geig(A, B, ev, X) : clg::dense::eig(A, ev, X);
  if (!ok) return CLG_ERR_BREAKDOWN;
  for (int i = 0; i < n; ++i) {
    w[2 * i] = ev[i].real();
    w[2 * i + 1] = ev[i].imag();
  }
  for (int i = 0; i < n * n; ++i) {
    x[2 * i] = X.a[i].real();
    x[2 * i + 1] = X.a[i].imag();
  }
  return CLG_SUCCESS;
}

}  // extern "C"
