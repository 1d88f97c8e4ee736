// Movie stack files on the host: MRC, MRC-gz and strip TIFF behind one
// handle (mc_stack_*).  Replaces the readers MRC, MRCZ and MRCT
// (mrc.cpp:29-157, 325-382; mrcz.cpp:23-110; mrct.cpp:29-152) and the format
// detection of the alignment thread (DFAlign.cu:470-479 with isTIFF, isMRCZ
// and isMRC, func.cpp:557-627).  Host code only: nothing here needs a GPU.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mc.h"
#include "tiff_read.h"

namespace mc {
int record_error(int code, const char* text);  // mc_plan.cu: sets mc_last_error()
}

namespace {

// Offsets of the MRC header fields this reader needs (struct MRCHeader,
// mrcheader.h:3-45): nx, ny, nz, mode at 0..15, nsymbt at 92, map at 208.
constexpr int kHdrBytes = 1024;

int32_t hdr_i32(const unsigned char* h, int off) {
  int32_t v;
  std::memcpy(&v, h + off, 4);
  return v;
}

bool has_map_stamp(const unsigned char* h) { return std::memcmp(h + 208, "MAP ", 4) == 0; }

// IEEE-754 binary16 -> binary32 (exact: every half is a float): sign,
// 5-bit exponent (bias 15), 10-bit fraction; subnormals scaled by 2^-24.
float half_bits_to_float(uint16_t h) {
  const int sign = h >> 15, e = (h >> 10) & 31, f = h & 1023;
  float v;
  if (e == 0) v = std::ldexp((float)f, -24);
  else if (e == 31) v = f ? std::numeric_limits<float>::quiet_NaN() : std::numeric_limits<float>::infinity();
  else v = std::ldexp((float)(f | 1024), e - 25);
  return sign ? -v : v;
}

// MRC::getWordLength (mrc.cpp:99-118) for the modes a plan decodes.
int word_length(int mode) {
  switch (mode) {
    case 0: return 1;
    case 1: return 2;
    case 2: return 4;
    case 6: return 2;
    case MC_MODE_U8: return 1;
    case MC_MODE_F16: return 2;  // MRC2014 mode 12 (IEEE half); the reference reads no such files
    default: return 0;
  }
}

int fail(int code, const std::string& what) { return mc::record_error(code, what.c_str()); }

bool first_two(const char* path, int& a, int& b) {
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return false;
  a = std::fgetc(fp);
  b = std::fgetc(fp);
  std::fclose(fp);
  return true;
}

}  // namespace

struct mc_stack {
  mc_stack_info info{};
  long long data_offset = 0;  // 1024 + nsymbt for MRC and MRC-gz
  FILE* fp = nullptr;
  gzFile gz = nullptr;
  std::unique_ptr<mc::TiffFile> tiff;
  std::mutex mu;  // one reader of fp/gz at a time

  ~mc_stack() {
    if (fp) std::fclose(fp);
    if (gz) gzclose(gz);
  }
  size_t frame_bytes() const { return (size_t)info.nx * info.ny * word_length(info.mode); }
};

extern "C" {

int mc_stack_open(const char* path, mc_stack** out) {
  if (!path || !out) return fail(MC_E_ARG, "mc_stack_open: null argument");
  *out = nullptr;
  int a = -1, b = -1;
  if (!first_two(path, a, b)) return fail(MC_E_IO, std::string("cannot open ") + path);
  std::unique_ptr<mc_stack> s(new mc_stack);
  // isTIFF: the byte-order mark alone picks the TIFF reader
  if ((a == 'I' && b == 'I') || (a == 'M' && b == 'M')) {
    s->tiff.reset(new mc::TiffFile);
    std::string err;
    if (!s->tiff->open(path, err)) return fail(MC_E_IO, std::string(path) + ": TIFF: " + err);
    const mc::TiffDir& d = s->tiff->dir(0);
    s->info.nx = (int)d.width;
    s->info.ny = (int)d.length;
    s->info.nz = s->tiff->ndirs();
    s->info.mode = d.bits == 8 ? MC_MODE_U8 : 6;
    s->info.file_mode = 7199;  // fakeReadHeader (mrct.cpp:104-123)
    s->info.format = MC_STACK_TIFF;
    s->info.bits = (int)d.bits;
    s->info.compression = (int)d.compression;
    *out = s.release();
    return MC_OK;
  }
  unsigned char h[kHdrBytes];
  // isMRCZ: the gzip magic and a 'MAP ' stamp in the inflated header
  if (a == 0x1f && b == 0x8b) {
    gzFile gz = gzopen(path, "rb");
    if (gz && gzread(gz, h, kHdrBytes) == kHdrBytes && has_map_stamp(h)) {
      gzbuffer(gz, 1 << 20);
      s->gz = gz;
      s->info.format = MC_STACK_MRCZ;
    } else if (gz) {
      gzclose(gz);
    }
  }
  // isMRC: the stamp, or a file name that contains "mrc"
  if (!s->gz) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(MC_E_IO, std::string("cannot open ") + path);
    const bool full = std::fread(h, 1, kHdrBytes, fp) == (size_t)kHdrBytes;
    if (!full || !(has_map_stamp(h) || std::strstr(path, "mrc") != nullptr)) {
      std::fclose(fp);
      return fail(MC_E_IO, std::string(path) + ": Only MRC, MRC-gz, TIFF file formats are supported.");
    }
    s->fp = fp;
    s->info.format = MC_STACK_MRC;
  }
  s->info.nx = hdr_i32(h, 0);
  s->info.ny = hdr_i32(h, 4);
  s->info.nz = hdr_i32(h, 8);
  s->info.mode = s->info.file_mode = hdr_i32(h, 12);
  s->info.compression = 0;
  s->data_offset = kHdrBytes + (long long)std::max(0, hdr_i32(h, 92));
  const int wl = word_length(s->info.mode);
  s->info.bits = 8 * wl;
  if (wl == 0 || s->info.mode == MC_MODE_U8)
    return fail(MC_E_IO, std::string(path) + ": unsupported MRC mode " + std::to_string(s->info.mode));
  if (s->info.nx <= 0 || s->info.ny <= 0 || s->info.nz <= 0)
    return fail(MC_E_IO, std::string(path) + ": header has no image geometry");
  *out = s.release();
  return MC_OK;
}

int mc_stack_get_info(const mc_stack* s, mc_stack_info* info) {
  if (!s || !info) return fail(MC_E_ARG, "mc_stack_get_info: null argument");
  *info = s->info;
  return MC_OK;
}

int mc_stack_read_frames(mc_stack* s, void* dst, int first, int count, int* got) {
  if (got) *got = 0;
  if (!s || (!dst && count > 0)) return fail(MC_E_ARG, "mc_stack_read_frames: null argument");
  if (first < 0 || count < 0 || (long long)first + count > s->info.nz)
    return fail(MC_E_ARG, "mc_stack_read_frames: frames outside the stack");
  if (count == 0) return MC_OK;
  const size_t fb = s->frame_bytes();
  unsigned char* out = static_cast<unsigned char*>(dst);
  int n_ok = 0;
  std::string err;
  if (s->info.format == MC_STACK_TIFF) {
    // directories decode independently: frames in parallel on host threads
    std::vector<char> ok(count, 0);
    std::vector<std::string> errs(count);
    const int nthreads = std::max(1, std::min<int>(count, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next{0};
    auto work = [&]() {
      for (int k = next++; k < count; k = next++)
        ok[k] = s->tiff->read_image(first + k, out + (size_t)k * fb, errs[k]) ? 1 : 0;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    while (n_ok < count && ok[n_ok]) n_ok++;
    if (n_ok < count) err = errs[n_ok];
  } else {
    std::lock_guard<std::mutex> lock(s->mu);
    const long long off = s->data_offset + (long long)first * (long long)fb;
    if (s->info.format == MC_STACK_MRC) {
      if (fseeko(s->fp, (off_t)off, SEEK_SET) == 0) n_ok = (int)(std::fread(out, 1, fb * count, s->fp) / fb);
    } else {
      // gzseek forward inflates and discards; backward rewinds (mrcz.cpp:103-109)
      if (gzseek(s->gz, (z_off_t)off, SEEK_SET) == (z_off_t)off) {
        for (; n_ok < count; n_ok++) {
          const int r = gzread(s->gz, out + (size_t)n_ok * fb, (unsigned)fb);
          if (r != (int)fb) break;
        }
      }
    }
    if (n_ok < count) err = "short read";
  }
  if (got) *got = n_ok;
  if (n_ok < count) return fail(MC_E_IO, "frame " + std::to_string(first + n_ok) + ": " + err);
  return MC_OK;
}

int mc_stack_read_frame_float(mc_stack* s, float* dst, int n) {
  if (!s || !dst) return fail(MC_E_ARG, "mc_stack_read_frame_float: null argument");
  const size_t npx = (size_t)s->info.nx * s->info.ny;
  std::vector<unsigned char> raw(s->frame_bytes());
  const int rc = mc_stack_read_frames(s, raw.data(), n, 1, nullptr);
  if (rc != MC_OK) return rc;
  switch (s->info.mode) {
    case 0:
      for (size_t i = 0; i < npx; i++) dst[i] = (float)((const signed char*)raw.data())[i];
      break;
    case MC_MODE_U8:
      for (size_t i = 0; i < npx; i++) dst[i] = (float)raw[i];
      break;
    case 1:
      for (size_t i = 0; i < npx; i++) dst[i] = (float)((const int16_t*)raw.data())[i];
      break;
    case 6:
      for (size_t i = 0; i < npx; i++) dst[i] = (float)((const uint16_t*)raw.data())[i];
      break;
    case MC_MODE_F16:
      for (size_t i = 0; i < npx; i++) dst[i] = half_bits_to_float(((const uint16_t*)raw.data())[i]);
      break;
    default:
      std::memcpy(dst, raw.data(), npx * sizeof(float));
      break;
  }
  return MC_OK;
}

void mc_stack_close(mc_stack* s) { delete s; }

}  // extern "C"
