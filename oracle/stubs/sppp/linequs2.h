/* Test infrastructure: a project-written stand-in for the small part of the
 * SP++ 3.0 signal-processing library (namespace splab, header linequs2.h)
 * that the reference's DFAlign.cu and mfunc.h call.  SP++ itself is not
 * vendored with the reference (README.md names it without a version) and is
 * not installed here; this header lets the reference's alignment code
 * compile from its own sources so that it can be run as a parity pin and as
 * the timed "reference cuFFT build".  Nothing in the product links it.
 *
 * Written from the mathematics, not from SP++'s sources:
 *   Matrix<T>, Vector<T>   dense row-major storage; m[i] is a pointer to
 *                          row i, getRow/setRow copy one row
 *   operator*, operator-, abs, sum   the usual matrix-vector algebra
 *   lsSolver(A, b)         least squares min ||A x - b||_2 of a full-column-
 *                          rank A by Householder QR (Golub & Van Loan,
 *                          "Matrix Computations", 4th ed., Alg. 5.2.1 and
 *                          section 5.3.3), complex arithmetic in FP64
 *   PI                     the constant pi
 *   CSVD<R>::dec / rank    singular values of a complex matrix by the one-
 *                          sided Jacobi method of Hestenes (1958), as in
 *                          Demmel & Veselic (1992); rank = number of singular
 *                          values above max(m, n) * s_max * DBL_EPSILON
 *
 * Call sites in the reference: DFAlign.cu:877-948 (A, b, lsSolver, abs,
 * sum), mfunc.h:50-146 (Matrix construction, OD_Threshold's getRow/setRow
 * and CSVD rank test). */
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstddef>
#include <vector>

namespace splab {

// SP++ exports the constant pi; DFAlign.cu:224 uses it as PI.
const double PI = 3.14159265358979323846;

template <typename T>
class Vector {
 public:
  Vector() {}
  explicit Vector(int n) : v_((size_t)std::max(n, 0), T()) {}
  Vector(int n, const T& init) : v_((size_t)std::max(n, 0), init) {}
  int size() const { return (int)v_.size(); }
  int dim() const { return size(); }
  T& operator[](int i) { return v_[(size_t)i]; }
  const T& operator[](int i) const { return v_[(size_t)i]; }
  T& operator()(int i) { return v_[(size_t)i - 1]; }  // SP++ also offers 1-based access

 private:
  std::vector<T> v_;
};

template <typename T>
class Matrix {
 public:
  Matrix() : r_(0), c_(0) {}
  Matrix(int rows, int cols) : r_(rows), c_(cols), a_((size_t)rows * cols, T()) {}
  Matrix(int rows, int cols, const T& init) : r_(rows), c_(cols), a_((size_t)rows * cols, init) {}
  int rows() const { return r_; }
  int cols() const { return c_; }
  T* operator[](int i) { return a_.data() + (size_t)i * c_; }
  const T* operator[](int i) const { return a_.data() + (size_t)i * c_; }
  T& operator()(int i, int j) { return a_[(size_t)(i - 1) * c_ + (j - 1)]; }
  Vector<T> getRow(int i) const {
    Vector<T> r(c_);
    for (int j = 0; j < c_; j++) r[j] = (*this)[i][j];
    return r;
  }
  void setRow(const Vector<T>& v, int i) {
    for (int j = 0; j < c_ && j < v.size(); j++) (*this)[i][j] = v[j];
  }
  Vector<T> getColumn(int j) const {
    Vector<T> c(r_);
    for (int i = 0; i < r_; i++) c[i] = (*this)[i][j];
    return c;
  }
  void setColumn(const Vector<T>& v, int j) {
    for (int i = 0; i < r_ && i < v.size(); i++) (*this)[i][j] = v[i];
  }

 private:
  int r_, c_;
  std::vector<T> a_;
};

template <typename T>
Vector<T> operator*(const Matrix<T>& A, const Vector<T>& x) {
  Vector<T> y(A.rows(), T());
  for (int i = 0; i < A.rows(); i++) {
    T s = T();
    for (int j = 0; j < A.cols(); j++) s += A[i][j] * x[j];
    y[i] = s;
  }
  return y;
}

template <typename T>
Vector<T> operator-(const Vector<T>& a, const Vector<T>& b) {
  Vector<T> r(a.size());
  for (int i = 0; i < a.size(); i++) r[i] = a[i] - b[i];
  return r;
}

template <typename T>
Vector<T> operator+(const Vector<T>& a, const Vector<T>& b) {
  Vector<T> r(a.size());
  for (int i = 0; i < a.size(); i++) r[i] = a[i] + b[i];
  return r;
}

template <typename R>
Vector<R> abs(const Vector<std::complex<R> >& v) {
  Vector<R> r(v.size());
  for (int i = 0; i < v.size(); i++) r[i] = std::abs(v[i]);
  return r;
}

template <typename T>
T sum(const Vector<T>& v) {
  T s = T();
  for (int i = 0; i < v.size(); i++) s += v[i];
  return s;
}

namespace detail {
inline double conj_if(double x) { return x; }
inline std::complex<double> conj_if(const std::complex<double>& z) { return std::conj(z); }
inline double sq(double x) { return x * x; }
inline double sq(const std::complex<double>& z) { return std::norm(z); }
}  // namespace detail

/* Householder QR least squares of a tall, full-column-rank A: Q^H A = R,
 * x = R^{-1} (Q^H b)[0:n].  Each reflector H = I - tau v v^H maps column k
 * below the diagonal onto -e^{i arg(a_kk)} ||a|| e_k. */
template <typename T>
Vector<T> lsSolver(const Matrix<T>& A0, const Vector<T>& b0) {
  const int m = A0.rows(), n = A0.cols();
  Matrix<T> A = A0;
  Vector<T> b = b0;
  for (int k = 0; k < n && k < m; k++) {
    double nrm2 = 0.0;
    for (int i = k; i < m; i++) nrm2 += detail::sq(A[i][k]);
    const double nrm = std::sqrt(nrm2);
    if (nrm == 0.0) continue;
    const T akk = A[k][k];
    const double aabs = std::abs(akk);
    const T phase = aabs > 0.0 ? akk / aabs : T(1.0);
    const T alpha = -phase * nrm;  // new diagonal entry
    // v = x - alpha e_k, stored in column k (v_k = akk - alpha)
    std::vector<T> v((size_t)(m - k));
    v[0] = akk - alpha;
    for (int i = k + 1; i < m; i++) v[(size_t)(i - k)] = A[i][k];
    double vv = 0.0;
    for (size_t i = 0; i < v.size(); i++) vv += detail::sq(v[i]);
    if (vv == 0.0) continue;
    const double tau = 2.0 / vv;
    // apply H to the remaining columns and to b
    for (int j = k; j < n; j++) {
      T s = T();
      for (int i = k; i < m; i++) s += detail::conj_if(v[(size_t)(i - k)]) * A[i][j];
      s *= tau;
      for (int i = k; i < m; i++) A[i][j] -= v[(size_t)(i - k)] * s;
    }
    T s = T();
    for (int i = k; i < m; i++) s += detail::conj_if(v[(size_t)(i - k)]) * b[i];
    s *= tau;
    for (int i = k; i < m; i++) b[i] -= v[(size_t)(i - k)] * s;
  }
  // back substitution R x = (Q^H b)[0:n]
  Vector<T> x(n, T());
  for (int i = std::min(n, m) - 1; i >= 0; i--) {
    T s = b[i];
    for (int j = i + 1; j < n; j++) s -= A[i][j] * x[j];
    x[i] = A[i][i] != T() ? s / A[i][i] : T();
  }
  return x;
}

/* Singular values of a complex m x n matrix by one-sided Jacobi rotations of
 * its columns until every pair is orthogonal to working precision; the
 * singular values are the final column norms. */
template <typename R>
class CSVD {
 public:
  void dec(const Matrix<std::complex<R> >& A) {
    typedef std::complex<R> C;
    const int m = A.rows(), n = A.cols();
    std::vector<std::vector<C> > col((size_t)n, std::vector<C>((size_t)m));
    for (int j = 0; j < n; j++)
      for (int i = 0; i < m; i++) col[(size_t)j][(size_t)i] = A[i][j];
    const R tol = (R)(m > 0 ? m : 1) * (R)DBL_EPSILON;
    for (int sweep = 0; sweep < 60; sweep++) {
      bool rotated = false;
      for (int p = 0; p < n - 1; p++)
        for (int q = p + 1; q < n; q++) {
          R alpha = 0, beta = 0;
          C gamma = 0;
          for (int i = 0; i < m; i++) {
            alpha += std::norm(col[(size_t)p][(size_t)i]);
            beta += std::norm(col[(size_t)q][(size_t)i]);
            gamma += std::conj(col[(size_t)p][(size_t)i]) * col[(size_t)q][(size_t)i];
          }
          const R g = std::abs(gamma);
          if (g == 0 || g <= tol * std::sqrt(alpha * beta)) continue;
          rotated = true;
          // rotation of the Hermitian 2x2 Gram block [[alpha, gamma], [conj(gamma), beta]]
          const C ph = gamma / g;
          const R zeta = (beta - alpha) / (2 * g);
          const R t = (zeta >= 0 ? 1 : -1) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
          const R c = 1 / std::sqrt(1 + t * t), s = c * t;
          for (int i = 0; i < m; i++) {
            const C xp = col[(size_t)p][(size_t)i], xq = col[(size_t)q][(size_t)i];
            col[(size_t)p][(size_t)i] = c * xp - s * std::conj(ph) * xq;
            col[(size_t)q][(size_t)i] = s * ph * xp + c * xq;
          }
        }
      if (!rotated) break;
    }
    sv_.assign((size_t)n, 0);
    for (int j = 0; j < n; j++) {
      R s = 0;
      for (int i = 0; i < m; i++) s += std::norm(col[(size_t)j][(size_t)i]);
      sv_[(size_t)j] = std::sqrt(s);
    }
    std::sort(sv_.begin(), sv_.end(), [](R a, R b) { return a > b; });
    m_ = m;
    n_ = n;
  }
  int rank() const {
    if (sv_.empty()) return 0;
    const R thr = (R)std::max(m_, n_) * sv_[0] * (R)DBL_EPSILON;
    int r = 0;
    for (R s : sv_)
      if (s > thr) r++;
    return r;
  }
  Vector<R> getSV() const {
    Vector<R> v((int)sv_.size());
    for (size_t i = 0; i < sv_.size(); i++) v[(int)i] = sv_[i];
    return v;
  }

 private:
  std::vector<R> sv_;
  int m_ = 0, n_ = 0;
};

}  // namespace splab
