// Test-infrastructure driver around FFT-free functions of the reference's
// func.cpp (compiled from the reference tree by oracle/build_ref.sh against
// the stand-in headers in oracle/stubs/; never shipped).
//
//   ref_func cropsize <nx> <ny> <offx> <offy> <nsamout> <bin>       verifyCropSize (func.cpp:80-103)
//   ref_func crop2fft <in.f32> <nx> <ny> <offx> <offy> <nsamout> <bin> <out.f32>   (func.cpp:157-173)
//   ref_func cosmask  <nsam> <out.c64>                              cosmask2d on ones (func.cpp:348-370)
//   ref_func hist     <in.f32> <size> <threshold>                   histMinMax (func.cpp:372-420)
//   ref_func dispshort <in.f32> <size> <out.i16>                    buf2DispShort (func.cpp:441-456)
//   ref_func moddisp  <in.f32> <nsam> <out.f32>                     FFTModulusToDispBuf (func.cpp:459-489)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fftw3.h"
#include "func.h"

// func.cpp's FFT helpers link against these; none of the commands reaches them
fftwf_plan fftwf_plan_dft_r2c_2d(int, int, float*, fftwf_complex*, unsigned) { abort(); }
fftwf_plan fftwf_plan_dft_c2r_2d(int, int, fftwf_complex*, float*, unsigned) { abort(); }
void fftwf_execute(const fftwf_plan) { abort(); }
void fftwf_destroy_plan(fftwf_plan) { abort(); }

template <typename T>
static std::vector<T> load(const char* path, size_t n) {
  std::vector<T> v(n);
  FILE* f = fopen(path, "rb");
  if (!f || fread(v.data(), sizeof(T), n, f) != n) exit(3);
  fclose(f);
  return v;
}
template <typename T>
static void save(const char* path, const T* p, size_t n) {
  FILE* f = fopen(path, "wb");
  if (!f) exit(4);
  fwrite(p, sizeof(T), n, f);
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const char* c = argv[1];
  if (!strcmp(c, "cropsize") && argc == 8) {
    printf("%d\n", verifyCropSize(atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]),
                                  (float)atof(argv[7])));
    return 0;
  }
  if (!strcmp(c, "crop2fft") && argc == 10) {
    const int nx = atoi(argv[3]), ny = atoi(argv[4]);
    std::vector<float> in = load<float>(argv[2], (size_t)nx * ny);
    const int ns = verifyCropSize(nx, ny, atoi(argv[5]), atoi(argv[6]), atoi(argv[7]), (float)atof(argv[8]));
    std::vector<float> out((size_t)(ns + 2) * (ns > 0 ? ns : 1), 0.f);
    const int r = crop2fft(in.data(), nx, ny, out.data(), atoi(argv[5]), atoi(argv[6]), atoi(argv[7]),
                           (float)atof(argv[8]));
    save(argv[9], out.data(), out.size());
    printf("%d\n", r);
    return 0;
  }
  if (!strcmp(c, "cosmask") && argc == 4) {
    const int n = atoi(argv[2]);
    std::vector<std::complex<float> > v((size_t)(n / 2 + 1) * n, std::complex<float>(1.f, 1.f));
    cosmask2d(v.data(), n);
    save(argv[3], v.data(), v.size());
    return 0;
  }
  if (!strcmp(c, "hist") && argc == 5) {
    const int n = atoi(argv[3]);
    std::vector<float> in = load<float>(argv[2], n);
    float mn, mx;
    histMinMax(in.data(), n, mn, mx, (float)atof(argv[4]));
    printf("%.9g %.9g\n", mn, mx);
    return 0;
  }
  if (!strcmp(c, "dispshort") && argc == 5) {
    const int n = atoi(argv[3]);
    std::vector<float> in = load<float>(argv[2], n);
    std::vector<short> out(n);
    buf2DispShort(out.data(), in.data(), n);
    save(argv[4], out.data(), out.size());
    return 0;
  }
  if (!strcmp(c, "moddisp") && argc == 5) {
    const int n = atoi(argv[3]);
    std::vector<float> in = load<float>(argv[2], (size_t)n * (n / 2 + 1));
    std::vector<float> out((size_t)n * (n + 2), 0.f);
    FFTModulusToDispBuf(in.data(), out.data(), n);
    save(argv[4], out.data(), out.size());
    return 0;
  }
  return 2;
}
