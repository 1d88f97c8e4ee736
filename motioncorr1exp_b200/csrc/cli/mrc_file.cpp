#include "mrc_file.h"

#include <cstring>
#include <vector>

int mrc_word_length(int mode) {
  switch (mode) {
    case 0: return 1;
    case 1: return 2;
    case 2: return 4;
    case 3: return 4;
    case 4: return 8;
    case 6: return 2;
    default: return 0;
  }
}

MrcStack::~MrcStack() { close(); }

void MrcStack::close() {
  if (fp_) fclose(fp_);
  fp_ = nullptr;
}

int MrcStack::open(const char* path) {
  close();
  fp_ = fopen(path, "rb");
  if (!fp_) return 0;
  if (fread(&h_, 1, 1024, fp_) < 1024) return -1;
  return 1;
}

size_t MrcStack::frame_bytes() const {
  return (size_t)h_.nx * (size_t)h_.ny * (size_t)mrc_word_length(h_.mode);
}

int MrcStack::read_frames(void* dst, int first, int count) {
  if (!fp_ || count <= 0) return 0;
  const size_t im = frame_bytes();
  const long long off = 1024LL + h_.nsymbt + (long long)first * (long long)im;
  if (fseeko(fp_, (off_t)off, SEEK_SET) != 0) return 0;
  const size_t got = fread(dst, 1, im * (size_t)count, fp_);
  return (int)(got / im);
}

bool MrcStack::read_frame_float(float* dst, int n) {
  const size_t npx = (size_t)h_.nx * h_.ny;
  std::vector<unsigned char> raw(frame_bytes());
  if (read_frames(raw.data(), n, 1) != 1) return false;
  switch (h_.mode) {
    case 0:
      for (size_t i = 0; i < npx; i++) dst[i] = (float)((const signed char*)raw.data())[i];
      break;
    case 1:
      for (size_t i = 0; i < npx; i++) dst[i] = (float)((const int16_t*)raw.data())[i];
      break;
    case 6:
      for (size_t i = 0; i < npx; i++) dst[i] = (float)((const uint16_t*)raw.data())[i];
      break;
    default:
      std::memcpy(dst, raw.data(), npx * sizeof(float));
      break;
  }
  return true;
}

bool is_mrc(const char* path, bool verb) {
  MrcStack s;
  if (s.open(path) > 0) {
    const MrcHeader& h = s.header();
    if (h.map[0] == 'M' && h.map[1] == 'A' && h.map[2] == 'P' && h.map[3] == ' ') {
      printf("Auto-detected file format: MRC2000\n");
      return true;
    }
    if (std::strstr(path, "mrc") != nullptr) {
      if (verb) printf("Auto-detected file format: old MRC with mrc extension.\n");
      return true;
    }
  }
  return false;
}

static bool first_two(const char* path, int& a, int& b) {
  FILE* fp = fopen(path, "rb");
  if (!fp) return false;
  a = fgetc(fp);
  b = fgetc(fp);
  fclose(fp);
  return true;
}

bool starts_with_gzip(const char* path) {
  int a, b;
  return first_two(path, a, b) && a == 0x1f && b == 0x8b;
}

bool starts_with_tiff(const char* path) {
  int a, b;
  return first_two(path, a, b) && ((a == 'I' && b == 'I') || (a == 'M' && b == 'M'));
}

bool write_mrc_float(const char* path, const float* data, int nx, int ny, int nz, MrcHeader* out_header) {
  MrcHeader h;
  std::memset(&h, 0, sizeof(h));
  h.nx = nx;
  h.ny = ny;
  h.nz = nz;
  h.mode = 2;
  h.cellb[0] = h.cellb[1] = h.cellb[2] = 90;
  h.mapc = 1;
  h.mapr = 2;
  h.maps = 3;
  const size_t size = (size_t)nx * ny * nz;
  float mn = size ? data[0] : 0.f, mx = mn;
  double mean = 0;
  for (size_t i = 0; i < size; i++) {
    if (mn > data[i]) mn = data[i];
    if (mx < data[i]) mx = data[i];
    mean += data[i];
  }
  if (size) mean /= (double)size;
  h.dmin = mn;
  h.dmax = mx;
  h.dmean = (float)mean;
  FILE* fp = fopen(path, "wb");
  if (!fp) return false;
  bool ok = fwrite(&h, 1, 1024, fp) == 1024;
  ok = ok && fwrite(data, sizeof(float), size, fp) == size;
  ok = (fclose(fp) == 0) && ok;
  if (out_header) *out_header = h;
  return ok;
}

bool write_mrc_short(const char* path, const int16_t* data, int nx, int ny, int nz) {
  MrcHeader h;
  std::memset(&h, 0, sizeof(h));
  h.nx = nx;
  h.ny = ny;
  h.nz = nz;
  h.mode = 1;
  h.cellb[0] = h.cellb[1] = h.cellb[2] = 90;
  h.mapc = 1;
  h.mapr = 2;
  h.maps = 3;
  const size_t size = (size_t)nx * ny * nz;
  int16_t mn = size ? data[0] : 0, mx = mn;
  double mean = 0;
  for (size_t i = 0; i < size; i++) {
    if (mn > data[i]) mn = data[i];
    if (mx < data[i]) mx = data[i];
    mean += data[i];
  }
  if (size) mean /= (double)size;
  h.dmin = mn;
  h.dmax = mx;
  h.dmean = (float)mean;
  FILE* fp = fopen(path, "wb");
  if (!fp) return false;
  bool ok = fwrite(&h, 1, 1024, fp) == 1024;
  ok = ok && fwrite(data, sizeof(int16_t), size, fp) == size;
  return (fclose(fp) == 0) && ok;
}

MrcStackWriter::~MrcStackWriter() { close(); }

bool MrcStackWriter::open(const char* path, int nx, int ny, int nz) {
  close();
  fp_ = fopen(path, "wb");
  if (!fp_) return false;
  MrcHeader h;
  std::memset(&h, 0, sizeof(h));
  h.nx = nx;
  h.ny = ny;
  h.nz = nz;
  h.mode = 2;
  h.cellb[0] = h.cellb[1] = h.cellb[2] = 90;
  h.mapc = 1;
  h.mapr = 2;
  h.maps = 3;
  nx_ = nx;
  ny_ = ny;
  return fwrite(&h, 1, 1024, fp_) == 1024;
}

bool MrcStackWriter::write_frame(const float* data, int n) {
  if (!fp_ || n < 0) return false;
  const size_t bytes = (size_t)nx_ * ny_ * sizeof(float);
  if (fseeko(fp_, (off_t)(1024 + (size_t)n * bytes), SEEK_SET) != 0) return false;
  return fwrite(data, 1, bytes, fp_) == bytes;
}

bool MrcStackWriter::close() {
  if (!fp_) return true;
  const bool ok = fclose(fp_) == 0;
  fp_ = nullptr;
  return ok;
}
