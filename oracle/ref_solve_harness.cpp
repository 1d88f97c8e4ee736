// Test-infrastructure driver of the reference's own drift solve: mfunc.h
// (OD_SetEquation_All, OD_Threshold, Min_VectorIndex) compiled from the
// reference tree against the project's SP++ stand-in (oracle/stubs/sppp),
// running the steps of DFAlign.cu:875-948 on pair shifts read from stdin.
// Never shipped; used by tests/test_oracle.py to pin the oracle's
// least-squares solve and outlier rejection.
//
//   stdin : nframe fod kithresh, then npairs lines "sx sy" (npairs is
//           OD_GetNRow_All(nframe, fod); pairs in OD_SetEquation_All order)
//   stdout: "pairs P", P lines "i j"; "ki1" + P values; "good G" + G indices;
//           "ki2" + G values; "shift" + (nframe-1) lines "re im"
#include <cstdio>
#include <cstdlib>

#include "mfunc.h"

int main() {
  int nframe = 0, fod = 0;
  double kithresh = 0.0;
  if (scanf("%d %d %lf", &nframe, &fod, &kithresh) != 3) return 2;
  // DFAlign.cu:876-881
  Matrix<complex<double> > A;
  vector<complex<int> > list;
  const int ncomp = OD_SetEquation_All(A, list, nframe, fod);
  Vector<complex<double> > b = Vector<complex<double> >(ncomp);
  for (int j = 0; j < ncomp; j++) {
    double sx, sy;
    if (scanf("%lf %lf", &sx, &sy) != 2) return 3;
    b[j] = complex<double>(sx, sy);
  }
  // DFAlign.cu:914-948 (kiThresh is the float parameter widened to double)
  Vector<complex<double> > shift = lsSolver(A, b);
  Vector<double> ki = abs(A * shift - b);
  printf("pairs %d\n", ncomp);
  for (size_t j = 0; j < list.size(); j++) printf("%d %d\n", list[j].real(), list[j].imag());
  printf("ki1\n");
  for (int j = 0; j < ki.size(); j++) printf("%.17g\n", ki[j]);
  const double thr = (double)(float)kithresh;
  vector<int> goodlist = OD_Threshold(A, b, ki, thr);
  shift = lsSolver(A, b);
  ki = abs(A * shift - b);
  printf("good %d\n", (int)goodlist.size());
  for (size_t j = 0; j < goodlist.size(); j++) printf("%d\n", goodlist[j]);
  printf("ki2\n");
  for (int j = 0; j < ki.size(); j++) printf("%.17g\n", ki[j]);
  printf("shift\n");
  for (int j = 0; j < shift.size(); j++) printf("%.17g %.17g\n", shift[j].real(), shift[j].imag());
  return 0;
}
