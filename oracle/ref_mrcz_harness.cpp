// Test-infrastructure driver around the reference's own MRC-gz reader
// (mrcz.cpp on top of mrc.cpp, compiled from the reference tree by
// oracle/build_ref.sh with zlib; never shipped).
//
//   ref_mrcz read   <in.mrc.gz> <frame> <out.f32>   read2DIm_32bit through MRCZ::read2DIm (mrcz.cpp:103-109)
//   ref_mrcz header <in.mrc.gz>                     nx ny nz mode
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mrcz.h"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  MRCZ m;
  if (m.open(argv[2], "rb") <= 0) return 3;
  if (!strcmp(argv[1], "read") && argc == 5) {
    std::vector<float> d((size_t)m.getNx() * m.getNy());
    if (m.read2DIm_32bit(d.data(), atoi(argv[3])) <= 0) return 4;
    FILE* f = fopen(argv[4], "wb");
    if (!f) return 5;
    fwrite(d.data(), sizeof(float), d.size(), f);
    fclose(f);
    m.close();
    return 0;
  }
  if (!strcmp(argv[1], "header")) {
    printf("%d %d %d %d\n", m.getNx(), m.getNy(), m.getNz(), m.getMode());
    m.close();
    return 0;
  }
  return 2;
}
