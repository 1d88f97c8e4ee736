// Test-infrastructure driver of the reference's own pair stage (cufunc.cu
// and func.cpp compiled from the reference tree by oracle/build_ref.sh, FFTW
// replaced by the direct DFTs of oracle/ref_fftw_dft.cpp; never shipped).
// For frames already cropped to nsam x nsam it runs what ThreadFunc_cuAlign
// does per pair (DFAlign.cu:768-770, 882-900): cuFFT R2C of every frame in
// place on padded rows, MkPosList with the B-factor, then per pair
// GPUShiftCC(frame j, frame i), cuFFT C2R and FindShift.
//
//   ref_pair <frames.f32> <nz> <nsam|nu/nsam> <bfactor> <box> <nps> <pairs.i32> <npairs> <out.txt> <boxes.f32>
//            [<spectra.f32> [<sum.f64> <nsum> <image.f32>]]
//   out.txt: one line per pair "i j sx sy cc"
//   nu/nsam: frames of nu x nu transformed at nu and Fourier-cropped to nsam
//   by GPUMemBinD2D (DFAlign.cu:773-779)
//   spectra.f32: every frame's cuFFT R2C, (nsam/2+1) x nsam complex rows ky
//   sum.f64: nsum records (frame, sx, sy, apply) summed as DFAlign.cu:1142-1292
//   does (first frame shifted only when apply; even positions into one sum,
//   odd into the other, added; C2R, times 1/nsam^2); image.f32 nsam x nsam
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cufunc.h"
#include "func.h"

int main(int argc, char** argv) {
  if (argc != 11 && argc != 12 && argc != 15) return 2;
  const int nz = atoi(argv[2]), box = atoi(argv[5]), nps = atoi(argv[6]);
  int nu = atoi(argv[3]), nsam = nu;
  if (const char* sl = strchr(argv[3], '/')) nsam = atoi(sl + 1);
  const float bfactor = (float)atof(argv[4]);
  const int npairs = atoi(argv[8]);
  if (!initGPU(0)) return 3;
  const int sizeb = (nsam + 2) * nsam, sizec = (nsam / 2 + 1) * nsam, sizebu = (nu + 2) * nu;
  std::vector<float> frames((size_t)nz * nu * nu);
  FILE* f = fopen(argv[1], "rb");
  if (!f || fread(frames.data(), sizeof(float), frames.size(), f) != frames.size()) return 4;
  fclose(f);
  std::vector<int> pairs(2 * (size_t)npairs);
  f = fopen(argv[7], "rb");
  if (!f || fread(pairs.data(), sizeof(int), pairs.size(), f) != pairs.size()) return 5;
  fclose(f);
  float *dfft = 0, *dsum = 0, *dunb = 0;
  MASK* dPosList = 0;
  if (!GPUMemAlloc((void**)&dfft, sizeof(float) * sizeb) || !GPUMemAlloc((void**)&dsum, sizeof(float) * sizeb) ||
      !GPUMemAlloc((void**)&dunb, sizeof(float) * sizebu) || !GPUMemAlloc((void**)&dPosList, sizeof(MASK) * sizec))
    return 6;
  cufftHandle uplan = GPUFFTPlan(nu), iplan = GPUIFFTPlan(nsam);
  // forward transforms (crop2fft lays the rows out padded to nu + 2), then
  // the Fourier crop to nsam when binning
  std::vector<float> hbuf((size_t)nz * sizeb), pad(sizebu);
  for (int k = 0; k < nz; k++) {
    crop2fft(frames.data() + (size_t)k * nu * nu, nu, pad.data(), 0, 0, nu, 1.0f);
    GPUMemH2D(dunb, pad.data(), sizeof(float) * sizebu);
    GPUFFT2d(dunb, uplan);
    GPUSync();
    if (nu != nsam) GPUMemBinD2D(dfft, dunb, nsam, nu);
    else GPUMemD2D(dfft, dunb, sizeof(float) * sizeb);
    GPUSync();
    GPUMemD2H(hbuf.data() + (size_t)k * sizeb, dfft, sizeof(float) * sizeb);
  }
  std::vector<MASK> pos(sizec);
  MkPosList(pos.data(), nsam, bfactor);
  GPUMemH2D(dPosList, pos.data(), sizeof(MASK) * sizec);
  FILE* out = fopen(argv[9], "w");
  FILE* boxes = fopen(argv[10], "wb");
  if (!out || !boxes) return 7;
  std::vector<float> hbox((size_t)box * box);
  for (int p = 0; p < npairs; p++) {
    const int i = pairs[2 * p], j = pairs[2 * p + 1];
    GPUMemH2D(dsum, hbuf.data() + (size_t)i * sizeb, sizeof(float) * sizeb);
    GPUMemH2D(dfft, hbuf.data() + (size_t)j * sizeb, sizeof(float) * sizeb);
    GPUShiftCC(dfft, dsum, dPosList, 0, 0, nsam);
    GPUSync();
    GPUIFFT2d(dfft, iplan);
    GPUSync();
    float sx = 0, sy = 0;
    const float cc = FindShift(dfft, nsam, hbox.data(), box, sx, sy, nps - 1);
    fprintf(out, "%d %d %.9g %.9g %.9g\n", i, j, sx, sy, cc);
    fwrite(hbox.data(), sizeof(float), hbox.size(), boxes);
  }
  fclose(out);
  fclose(boxes);
  if (argc >= 12) {
    FILE* sp = fopen(argv[11], "wb");
    if (!sp) return 8;
    for (int k = 0; k < nz; k++) fwrite(hbuf.data() + (size_t)k * sizeb, sizeof(float), sizeb, sp);
    fclose(sp);
  }
  if (argc == 15) {
    const int nsum = atoi(argv[13]);
    std::vector<double> rec(4 * (size_t)nsum);
    FILE* sf = fopen(argv[12], "rb");
    if (!sf || fread(rec.data(), sizeof(double), rec.size(), sf) != rec.size()) return 9;
    fclose(sf);
    float* dsum2 = 0;
    if (!GPUMemAlloc((void**)&dsum2, sizeof(float) * sizeb)) return 10;
    GPUMemZero((void**)&dsum, sizeof(float) * sizeb);
    GPUMemZero((void**)&dsum2, sizeof(float) * sizeb);
    for (int q = 0; q < nsum; q++) {
      const int k = (int)rec[4 * q];
      GPUMemH2D(dfft, hbuf.data() + (size_t)k * sizeb, sizeof(float) * sizeb);
      if (rec[4 * q + 3] != 0.0) GPUShift(dfft, dPosList, (float)rec[4 * q + 1], (float)rec[4 * q + 2], nsam);
      GPUAdd((q & 1) ? dsum2 : dsum, dfft, sizeb);
      GPUSync();
    }
    GPUAdd(dsum, dsum2, sizeb);
    GPUIFFT2d(dsum, iplan);
    GPUMultiplyNum(dsum, (float)(1.0 / ((double)nsam * nsam)), sizeb);  // 1.0/size, size = nsam*nsam
    GPUSync();
    std::vector<float> img(sizeb), flat((size_t)nsam * nsam);
    GPUMemD2H(img.data(), dsum, sizeof(float) * sizeb);
    fft2buf(flat.data(), img.data(), nsam);
    FILE* im = fopen(argv[14], "wb");
    if (!im) return 11;
    fwrite(flat.data(), sizeof(float), flat.size(), im);
    fclose(im);
    GPUMemFree((void**)&dsum2);
  }
  GPUFFTDestroy(uplan);
  GPUFFTDestroy(iplan);
  GPUMemFree((void**)&dfft);
  GPUMemFree((void**)&dsum);
  GPUMemFree((void**)&dunb);
  GPUMemFree((void**)&dPosList);
  return 0;
}
