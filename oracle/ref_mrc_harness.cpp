// Test-infrastructure driver around the reference's own MRC class (mrc.cpp,
// compiled from the reference tree by oracle/build_ref.sh; never shipped).
//
//   ref_mrc write <out.mrc> <nx> <ny> <nz> <in.f32>   createMRC(float*) (mrc.cpp:243-274)
//   ref_mrc read  <in.mrc> <frame> <out.f32>           read2DIm_32bit (mrc.cpp:325-382)
//   ref_mrc header <in.mrc>                            nx ny nz mode dmin dmax dmean
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mrc.h"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  if (!strcmp(argv[1], "write") && argc == 7) {
    const int nx = atoi(argv[3]), ny = atoi(argv[4]), nz = atoi(argv[5]);
    std::vector<float> d((size_t)nx * ny * nz);
    FILE* f = fopen(argv[6], "rb");
    if (!f || fread(d.data(), sizeof(float), d.size(), f) != d.size()) return 3;
    fclose(f);
    MRC m;
    m.open(argv[2], "wb");
    m.createMRC(d.data(), nx, ny, nz);
    m.close();
    return 0;
  }
  if (!strcmp(argv[1], "read") && argc == 5) {
    MRC m;
    if (m.open(argv[2], "rb") <= 0) return 3;
    std::vector<float> d((size_t)m.getNx() * m.getNy());
    if (m.read2DIm_32bit(d.data(), atoi(argv[3])) <= 0) return 4;
    FILE* f = fopen(argv[4], "wb");
    fwrite(d.data(), sizeof(float), d.size(), f);
    fclose(f);
    m.close();
    return 0;
  }
  if (!strcmp(argv[1], "header")) {
    MRC m;
    if (m.open(argv[2], "rb") <= 0) return 3;
    printf("%d %d %d %d %.9g %.9g %.9g\n", m.getNx(), m.getNy(), m.getNz(), m.getMode(), m.getMin(), m.getMax(),
           m.getMean());
    m.close();
    return 0;
  }
  return 2;
}
