// Test-infrastructure stand-in for the four FFTW calls of the reference's
// func.cpp (fft2d / ifft2d, in place on rows padded to 2 (n1/2 + 1) floats):
// the unnormalised 2-D DFTs computed directly in double, row-column, zero
// rows skipped.  r2c: X[k0][k1] = sum x[i][j] exp(-2 pi i (k0 i/n0 + k1 j/n1)),
// k1 <= n1/2.  c2r: a complex inverse along dimension 0, then the real
// inverse along dimension 1 (imaginary parts of its DC and Nyquist terms
// dropped), as for a Hermitian input; FindShift only hands it Hermitian
// spectra (cosmask2d zeroes the 16-point Nyquist row and column).
#include <cmath>
#include <complex>
#include <vector>

#include "fftw3.h"

struct fftwf_plan_s {
  int n0, n1, c2r;
  float* real;
  float* cplx;
};

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned) {
  return new fftwf_plan_s{n0, n1, 0, in, reinterpret_cast<float*>(out)};
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned) {
  return new fftwf_plan_s{n0, n1, 1, out, reinterpret_cast<float*>(in)};
}
void fftwf_destroy_plan(fftwf_plan p) { delete p; }

void fftwf_execute(const fftwf_plan p) {
  typedef std::complex<double> C;
  const int n0 = p->n0, n1 = p->n1, h = n1 / 2 + 1;
  const bool inplace = p->real == p->cplx;
  const int rs = inplace ? 2 * h : n1;  // real row stride
  const double tau = 2.0 * 3.14159265358979323846;
  // exp(-2 pi i m / n) for both lengths; w(m, n, +1) is the conjugate
  std::vector<C> t0(n0), t1(n1);
  for (int m = 0; m < n0; m++) t0[m] = std::polar(1.0, -tau * m / n0);
  for (int m = 0; m < n1; m++) t1[m] = std::polar(1.0, -tau * m / n1);
  auto w = [&](long long k, int n, double sgn) {
    const C v = (n == n0 ? t0 : t1)[(size_t)(k % n)];
    return sgn < 0 ? v : std::conj(v);
  };
  std::vector<C> a((size_t)n0 * h);
  if (!p->c2r) {
    for (int i = 0; i < n0; i++)
      for (int k1 = 0; k1 < h; k1++) {
        C s = 0;
        for (int j = 0; j < n1; j++) s += (double)p->real[(size_t)i * rs + j] * w((long long)k1 * j % n1, n1, -1.0);
        a[(size_t)i * h + k1] = s;
      }
    std::vector<C> b((size_t)n0 * h);
    for (int k1 = 0; k1 < h; k1++)
      for (int k0 = 0; k0 < n0; k0++) {
        C s = 0;
        for (int i = 0; i < n0; i++) s += a[(size_t)i * h + k1] * w((long long)k0 * i % n0, n0, -1.0);
        b[(size_t)k0 * h + k1] = s;
      }
    for (size_t q = 0; q < b.size(); q++) {
      p->cplx[2 * q] = (float)b[q].real();
      p->cplx[2 * q + 1] = (float)b[q].imag();
    }
    return;
  }
  std::vector<int> live;
  for (int k0 = 0; k0 < n0; k0++) {
    bool nz = false;
    for (int k1 = 0; k1 < h && !nz; k1++)
      nz = p->cplx[2 * ((size_t)k0 * h + k1)] != 0.f || p->cplx[2 * ((size_t)k0 * h + k1) + 1] != 0.f;
    if (nz) live.push_back(k0);
  }
  for (int i = 0; i < n0; i++)
    for (int k1 = 0; k1 < h; k1++) {
      C s = 0;
      for (int k0 : live)
        s += C(p->cplx[2 * ((size_t)k0 * h + k1)], p->cplx[2 * ((size_t)k0 * h + k1) + 1]) *
             w((long long)k0 * i % n0, n0, 1.0);
      a[(size_t)i * h + k1] = s;
    }
  std::vector<float> out((size_t)n0 * rs, 0.f);
  for (int i = 0; i < n0; i++)
    for (int j = 0; j < n1; j++) {
      double s = a[(size_t)i * h].real();
      if (n1 % 2 == 0) s += a[(size_t)i * h + n1 / 2].real() * ((j & 1) ? -1.0 : 1.0);
      for (int k1 = 1; k1 < (n1 + 1) / 2; k1++) s += 2.0 * (a[(size_t)i * h + k1] * w((long long)k1 * j % n1, n1, 1.0)).real();
      out[(size_t)i * rs + j] = (float)s;
    }
  for (size_t q = 0; q < out.size(); q++) p->real[q] = out[q];
}
