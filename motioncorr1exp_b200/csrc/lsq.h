// FP64 drift solve of the frame-pair system (host side, tiny: <= ~100 unknowns).
//
// Row r of the design matrix is the indicator of frame steps [i_r, j_r)
// (OD_SetEquation_All, mfunc.h:64-84); the right-hand side is the measured
// complex pair shift.  The solve uses FP64 normal equations + Cholesky; the
// rank test of OD_Threshold (mfunc.h:101-146) uses the identity
//   rank(A) = nframe - (connected components of the pair graph)
// which is exact for interval (difference) matrices.
#pragma once
#include <complex>
#include <utility>
#include <vector>

namespace mc {

using cplx = std::complex<double>;
using PairIJ = std::pair<int, int>;

// Least squares over the listed rows.  Returns false when A^T A is singular.
bool lsq_intervals(const std::vector<PairIJ>& rows, const std::vector<int>& use, int ncol,
                   const std::vector<cplx>& b, std::vector<cplx>& s);

// |A s - b| for the listed rows.
std::vector<double> lsq_residuals(const std::vector<PairIJ>& rows, const std::vector<int>& use,
                                  const std::vector<cplx>& b, const std::vector<cplx>& s);

// Rank of the rows in `use` (nframe - components).
int interval_rank(const std::vector<PairIJ>& rows, const std::vector<int>& use, int nframe);

// OD_Threshold: kept row indices, ascending.
std::vector<int> od_threshold(const std::vector<PairIJ>& rows, const std::vector<double>& ki, int nframe,
                              double kithresh);

}  // namespace mc
