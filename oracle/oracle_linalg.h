// Small dense linear algebra shared by the CPU oracles (test infrastructure
// only; see nddo_oracle.cpp and dftb_oracle.cpp).  Row-major N x N storage.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

namespace oracle_la {

// Neumaier-compensated running sum.  The NDDO energies are differences of
// sums over millions of terms that reach 1e5 Hartree for a few thousand AOs
// (E_el and E_rep cancel to 1e3); a plain running sum there loses 1e-8 to
// 1e-6 Hartree, above the precision the checks ask for.
struct CompensatedSum {
  double s = 0, c = 0;
  void add(double x) {
    const double t = s + x;
    c += std::fabs(s) >= std::fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  double value() const { return s + c; }
};

// Householder reduction of symmetric A to tridiagonal form; A is overwritten
// with the accumulated orthogonal transform Q (A_in = Q T Q^T); d = diagonal,
// e[i] = sub-diagonal T(i, i-1) for i >= 1.
inline void tridiagonalise(int n, std::vector<double>& a, std::vector<double>& d, std::vector<double>& e) {
  d.assign(n, 0);
  e.assign(n, 0);
  auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
  for (int i = n - 1; i > 0; --i) {
    int l = i - 1;
    double h = 0, scale = 0;
    if (l > 0) {
      for (int k = 0; k <= l; ++k) scale += std::fabs(A(i, k));
      if (scale == 0.0) {
        e[i] = A(i, l);
      } else {
        for (int k = 0; k <= l; ++k) {
          A(i, k) /= scale;
          h += A(i, k) * A(i, k);
        }
        double f = A(i, l);
        double g = f >= 0 ? -std::sqrt(h) : std::sqrt(h);
        e[i] = scale * g;
        h -= f * g;
        A(i, l) = f - g;
        f = 0;
        for (int j = 0; j <= l; ++j) {
          A(j, i) = A(i, j) / h;
          double gg = 0;
          for (int k = 0; k <= j; ++k) gg += A(j, k) * A(i, k);
          for (int k = j + 1; k <= l; ++k) gg += A(k, j) * A(i, k);
          e[j] = gg / h;
          f += e[j] * A(i, j);
        }
        double hh = f / (h + h);
        for (int j = 0; j <= l; ++j) {
          double ff = A(i, j);
          double gg = e[j] - hh * ff;
          e[j] = gg;
          for (int k = 0; k <= j; ++k) A(j, k) -= (ff * e[k] + gg * A(i, k));
        }
      }
    } else {
      e[i] = A(i, l);
    }
    d[i] = h;
  }
  d[0] = 0;
  e[0] = 0;
  for (int i = 0; i < n; ++i) {
    int l = i - 1;
    if (d[i] != 0.0) {
      for (int j = 0; j <= l; ++j) {
        double g = 0;
        for (int k = 0; k <= l; ++k) g += A(i, k) * A(k, j);
        for (int k = 0; k <= l; ++k) A(k, j) -= g * A(k, i);
      }
    }
    d[i] = A(i, i);
    A(i, i) = 1;
    for (int j = 0; j <= l; ++j) A(j, i) = A(i, j) = 0;
  }
}

// Implicit-shift QL on the tridiagonal (d, e) with eigenvector accumulation
// into z (columns).  Returns false if an eigenvalue fails to converge.
inline bool tridiagonal_ql(int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>& z) {
  for (int i = 1; i < n; ++i) e[i - 1] = e[i];
  if (n > 0) e[n - 1] = 0;
  auto Z = [&](int i, int j) -> double& { return z[(size_t)i * n + j]; };
  for (int l = 0; l < n; ++l) {
    int iter = 0, m;
    do {
      for (m = l; m < n - 1; ++m) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 1e-16 * dd) break;
      }
      if (m != l) {
        if (iter++ == 200) return false;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
        double s = 1, c = 1, p = 0;
        int i;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i], b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          for (int k = 0; k < n; ++k) {
            f = Z(k, i + 1);
            Z(k, i + 1) = s * Z(k, i) + c * f;
            Z(k, i) = c * Z(k, i) - s * f;
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0;
      }
    } while (m != l);
  }
  return true;
}

// Symmetric eigen-decomposition: eigenvalues ascending in w, eigenvectors in
// the columns of v (row-major N x N).
inline bool eigh(int n, const std::vector<double>& a, std::vector<double>& w, std::vector<double>& v) {
  v = a;
  std::vector<double> e;
  tridiagonalise(n, v, w, e);
  if (!tridiagonal_ql(n, w, e, v)) return false;
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return w[x] < w[y]; });
  std::vector<double> w2(n), v2((size_t)n * n);
  for (int j = 0; j < n; ++j) {
    w2[j] = w[order[j]];
    for (int i = 0; i < n; ++i) v2[(size_t)i * n + j] = v[(size_t)i * n + order[j]];
  }
  w.swap(w2);
  v.swap(v2);
  return true;
}

// Solve the small dense system M x = b by Gaussian elimination with partial pivoting.
inline bool solve_dense(int n, std::vector<double> M, std::vector<double>& b) {
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(M[r * n + c]) > std::fabs(M[piv * n + c])) piv = r;
    if (std::fabs(M[piv * n + c]) < 1e-300) return false;
    if (piv != c) {
      for (int k = 0; k < n; ++k) std::swap(M[c * n + k], M[piv * n + k]);
      std::swap(b[c], b[piv]);
    }
    for (int r = c + 1; r < n; ++r) {
      double f = M[r * n + c] / M[c * n + c];
      for (int k = c; k < n; ++k) M[r * n + k] -= f * M[c * n + k];
      b[r] -= f * b[c];
    }
  }
  for (int c = n - 1; c >= 0; --c) {
    double s = b[c];
    for (int k = c + 1; k < n; ++k) s -= M[c * n + k] * b[k];
    b[c] = s / M[c * n + c];
  }
  return true;
}


}  // namespace oracle_la
