#include "lsq.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace mc {

bool lsq_intervals(const std::vector<PairIJ>& rows, const std::vector<int>& use, int ncol,
                   const std::vector<cplx>& b, std::vector<cplx>& s) {
  // normal equations M s = A^T b; M[k][l] = #rows covering steps k and l
  std::vector<double> M((size_t)ncol * ncol, 0.0);
  std::vector<double> rr(ncol, 0.0), ri(ncol, 0.0);
  for (int r : use) {
    const int i = rows[r].first, j = rows[r].second;
    for (int k = i; k < j; k++) {
      rr[k] += b[r].real();
      ri[k] += b[r].imag();
      for (int l = i; l < j; l++) M[(size_t)k * ncol + l] += 1.0;
    }
  }
  // Cholesky M = L L^T (in place, lower triangle)
  double dmax = 0.0;
  for (int k = 0; k < ncol; k++) dmax = std::max(dmax, M[(size_t)k * ncol + k]);
  const double tiny = 1e-12 * std::max(dmax, 1.0);
  for (int k = 0; k < ncol; k++) {
    double d = M[(size_t)k * ncol + k];
    for (int m = 0; m < k; m++) d -= M[(size_t)k * ncol + m] * M[(size_t)k * ncol + m];
    if (!(d > tiny)) return false;
    const double lkk = std::sqrt(d);
    M[(size_t)k * ncol + k] = lkk;
    for (int i = k + 1; i < ncol; i++) {
      double v = M[(size_t)i * ncol + k];
      for (int m = 0; m < k; m++) v -= M[(size_t)i * ncol + m] * M[(size_t)k * ncol + m];
      M[(size_t)i * ncol + k] = v / lkk;
    }
  }
  // forward / back substitution for both right-hand sides
  std::vector<double> yr(ncol), yi(ncol);
  for (int i = 0; i < ncol; i++) {
    double vr = rr[i], vi = ri[i];
    for (int m = 0; m < i; m++) {
      vr -= M[(size_t)i * ncol + m] * yr[m];
      vi -= M[(size_t)i * ncol + m] * yi[m];
    }
    yr[i] = vr / M[(size_t)i * ncol + i];
    yi[i] = vi / M[(size_t)i * ncol + i];
  }
  s.assign(ncol, cplx(0.0, 0.0));
  for (int i = ncol - 1; i >= 0; i--) {
    double vr = yr[i], vi = yi[i];
    for (int m = i + 1; m < ncol; m++) {
      vr -= M[(size_t)m * ncol + i] * s[m].real();
      vi -= M[(size_t)m * ncol + i] * s[m].imag();
    }
    s[i] = cplx(vr / M[(size_t)i * ncol + i], vi / M[(size_t)i * ncol + i]);
  }
  return true;
}

std::vector<double> lsq_residuals(const std::vector<PairIJ>& rows, const std::vector<int>& use,
                                  const std::vector<cplx>& b, const std::vector<cplx>& s) {
  std::vector<double> ki;
  ki.reserve(use.size());
  for (int r : use) {
    cplx acc(0.0, 0.0);
    for (int k = rows[r].first; k < rows[r].second; k++) acc += s[k];
    ki.push_back(std::abs(acc - b[r]));
  }
  return ki;
}

namespace {
int find_root(std::vector<int>& par, int x) {
  while (par[x] != x) {
    par[x] = par[par[x]];
    x = par[x];
  }
  return x;
}
}  // namespace

int interval_rank(const std::vector<PairIJ>& rows, const std::vector<int>& use, int nframe) {
  std::vector<int> par(nframe);
  std::iota(par.begin(), par.end(), 0);
  int comps = nframe;
  for (int r : use) {
    const int a = find_root(par, rows[r].first), c = find_root(par, rows[r].second);
    if (a != c) {
      par[a] = c;
      comps--;
    }
  }
  return nframe - comps;
}

std::vector<int> od_threshold(const std::vector<PairIJ>& rows, const std::vector<double>& ki, int nframe,
                              double kithresh) {
  const int ncol = nframe - 1;
  const int nrow = (int)ki.size();
  // repeated first-minimum selection == stable ascending sort (mfunc.h:111-116)
  std::vector<int> order(nrow);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return ki[x] < ki[y]; });
  int i;
  for (i = nrow - 1; i >= ncol; i--)
    if (ki[order[i]] < kithresh) break;
  int ii = i;
  std::vector<int> good;
  int rank;
  do {
    good.assign(order.begin(), order.begin() + std::min(ii + 1, nrow));
    std::sort(good.begin(), good.end());
    rank = interval_rank(rows, good, nframe);
    ii++;
  } while (rank < ncol && ii < nrow);
  return good;
}

}  // namespace mc
