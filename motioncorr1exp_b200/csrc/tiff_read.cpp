// Strip-TIFF reader (see tiff_read.h).  Layout facts from the TIFF 6.0
// specification (header, IFD entries, StripOffsets/StripByteCounts,
// RowsPerStrip, LZW with 9..12-bit MSB-first codes and the early width
// change, PackBits, Predictor 2) and the BigTIFF extension (magic 43,
// 8-byte offsets and counts); Deflate streams are zlib streams.
#include "tiff_read.h"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <set>

namespace mc {
namespace {

enum : uint16_t {
  kWidth = 256,
  kLength = 257,
  kBits = 258,
  kCompression = 259,
  kStripOffsets = 273,
  kSpp = 277,
  kRowsPerStrip = 278,
  kStripByteCounts = 279,
  kPredictor = 317,
  kTileWidth = 322,
  kTileOffsets = 324,
};

bool pread_all(int fd, void* dst, size_t n, uint64_t off) {
  uint8_t* p = static_cast<uint8_t*>(dst);
  while (n > 0) {
    const ssize_t r = ::pread(fd, p, n, (off_t)off);
    if (r <= 0) return false;
    p += r;
    n -= (size_t)r;
    off += (uint64_t)r;
  }
  return true;
}

struct Endian {
  bool big;
  uint64_t get(const uint8_t* p, int bytes) const {
    uint64_t v = 0;
    if (big)
      for (int i = 0; i < bytes; i++) v = (v << 8) | p[i];
    else
      for (int i = bytes - 1; i >= 0; i--) v = (v << 8) | p[i];
    return v;
  }
};

int type_size(uint16_t type) {
  switch (type) {
    case 1: case 2: case 6: case 7: return 1;
    case 3: case 8: return 2;
    case 4: case 9: case 11: case 13: return 4;
    case 5: case 10: case 12: case 16: case 17: case 18: return 8;
    default: return 0;
  }
}

bool integer_type(uint16_t type) {
  return type == 1 || type == 3 || type == 4 || type == 13 || type == 16 || type == 18;
}

}  // namespace

// ------------------------------------------------------------------ codecs --
bool tiff_lzw_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t want) {
  // The pre-6.0 LSB-first variant starts with a zero byte and a set low bit.
  if (n >= 2 && src[0] == 0 && (src[1] & 1)) return false;
  constexpr int kMaxCodes = 4096;
  std::vector<uint16_t> prefix(kMaxCodes), len(kMaxCodes);
  std::vector<uint8_t> suffix(kMaxCodes), first(kMaxCodes);
  for (int i = 0; i < 256; i++) {
    prefix[i] = 0xffff;
    suffix[i] = first[i] = (uint8_t)i;
    len[i] = 1;
  }
  size_t out = 0, pos = 0;
  uint64_t acc = 0;
  int nacc = 0, width = 9, next = 258, old = -1;
  while (out < want) {
    while (nacc < width && pos < n) {
      acc = (acc << 8) | src[pos++];
      nacc += 8;
    }
    if (nacc < width) break;  // data exhausted without an end code
    const int code = (int)((acc >> (nacc - width)) & ((1u << width) - 1));
    nacc -= width;
    acc &= (nacc ? ((1ull << nacc) - 1) : 0);
    if (code == 257) break;
    if (code == 256) {
      width = 9;
      next = 258;
      old = -1;
      continue;
    }
    if (old < 0) {
      if (code > 255) return false;
      dst[out++] = (uint8_t)code;
      old = code;
      continue;
    }
    if (code > next) return false;
    if (next < kMaxCodes) {
      const uint8_t fb = code < next ? first[code] : first[old];
      prefix[next] = (uint16_t)old;
      suffix[next] = fb;
      first[next] = first[old];
      len[next] = (uint16_t)(len[old] + 1);
      next++;
      if (next >= (1 << width) - 1 && width < 12) width++;
    } else if (code == next) {
      return false;
    }
    const size_t L = len[code];
    int c = code;
    for (size_t k = L; k-- > 0;) {
      if (out + k < want) dst[out + k] = suffix[c];
      c = prefix[c];
    }
    out = std::min(out + L, want);
    old = code;
  }
  return out == want;
}

bool tiff_packbits_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t want) {
  size_t out = 0, pos = 0;
  while (out < want && pos < n) {
    const int c = (int8_t)src[pos++];
    if (c >= 0) {
      const size_t cnt = (size_t)c + 1;
      if (pos + cnt > n) return false;
      const size_t m = std::min(cnt, want - out);
      std::memcpy(dst + out, src + pos, m);
      out += m;
      pos += cnt;
    } else if (c != -128) {
      if (pos >= n) return false;
      const size_t m = std::min((size_t)(1 - c), want - out);
      std::memset(dst + out, src[pos++], m);
      out += m;
    }
  }
  return out == want;
}

bool tiff_deflate_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t want) {
  z_stream z;
  std::memset(&z, 0, sizeof(z));
  if (inflateInit(&z) != Z_OK) return false;
  z.next_in = const_cast<Bytef*>(src);
  z.avail_in = (uInt)n;
  z.next_out = dst;
  z.avail_out = (uInt)want;
  int r = Z_OK;
  while (z.avail_out > 0 && r == Z_OK) r = inflate(&z, Z_NO_FLUSH);
  const bool ok = z.total_out == want && (r == Z_OK || r == Z_STREAM_END || r == Z_BUF_ERROR);
  inflateEnd(&z);
  return ok;
}

// ------------------------------------------------------------------- file --
TiffFile::~TiffFile() {
  if (fd_ >= 0) ::close(fd_);
}

bool TiffFile::open(const char* path, std::string& err) {
  fd_ = ::open(path, O_RDONLY);
  if (fd_ < 0) {
    err = "cannot open file";
    return false;
  }
  struct stat st;
  if (fstat(fd_, &st) != 0) {
    err = "cannot stat file";
    return false;
  }
  file_size_ = (uint64_t)st.st_size;
  uint8_t hdr[16];
  if (file_size_ < 8 || !pread_all(fd_, hdr, std::min<uint64_t>(16, file_size_), 0)) {
    err = "file too short for a TIFF header";
    return false;
  }
  if (hdr[0] == 'I' && hdr[1] == 'I') big_endian_ = false;
  else if (hdr[0] == 'M' && hdr[1] == 'M') big_endian_ = true;
  else {
    err = "no TIFF byte-order mark";
    return false;
  }
  const Endian e{big_endian_};
  const uint64_t magic = e.get(hdr + 2, 2);
  bool bigtiff = false;
  uint64_t ifd = 0;
  if (magic == 42) {
    ifd = e.get(hdr + 4, 4);
  } else if (magic == 43 && file_size_ >= 16 && e.get(hdr + 4, 2) == 8) {
    bigtiff = true;
    ifd = e.get(hdr + 8, 8);
  } else {
    err = "not a classic TIFF or BigTIFF";
    return false;
  }
  const int cnt_bytes = bigtiff ? 8 : 2, entry_bytes = bigtiff ? 20 : 12, inline_bytes = bigtiff ? 8 : 4;
  std::set<uint64_t> seen;
  while (ifd != 0) {
    if (!seen.insert(ifd).second || seen.size() > (1u << 20)) {
      err = "directory chain loops";
      return false;
    }
    uint8_t cb[8];
    if (ifd + cnt_bytes > file_size_ || !pread_all(fd_, cb, cnt_bytes, ifd)) {
      err = "directory offset outside the file";
      return false;
    }
    const uint64_t nent = e.get(cb, cnt_bytes);
    if (nent == 0 || nent > 4096 || ifd + cnt_bytes + nent * entry_bytes + inline_bytes > file_size_) {
      err = "malformed directory";
      return false;
    }
    std::vector<uint8_t> ents(nent * entry_bytes + inline_bytes);
    if (!pread_all(fd_, ents.data(), ents.size(), ifd + cnt_bytes)) {
      err = "cannot read directory";
      return false;
    }
    TiffDir d;
    bool has_w = false, has_l = false, has_off = false, has_cnt = false;
    for (uint64_t k = 0; k < nent; k++) {
      const uint8_t* p = ents.data() + k * entry_bytes;
      const uint16_t tag = (uint16_t)e.get(p, 2), type = (uint16_t)e.get(p + 2, 2);
      const uint64_t count = e.get(p + 4, bigtiff ? 8 : 4);
      const uint8_t* vf = p + (bigtiff ? 12 : 8);
      if (tag == kTileWidth || tag == kTileOffsets) d.tiled = true;
      if (tag != kWidth && tag != kLength && tag != kBits && tag != kCompression && tag != kStripOffsets &&
          tag != kSpp && tag != kRowsPerStrip && tag != kStripByteCounts && tag != kPredictor)
        continue;
      const int ts = type_size(type);
      if (!integer_type(type) || count == 0 || count > (1u << 24)) {
        err = "unsupported field type or count for tag " + std::to_string(tag);
        return false;
      }
      std::vector<uint64_t> v(count);
      const uint64_t bytes = count * (uint64_t)ts;
      if (bytes <= (uint64_t)inline_bytes) {
        for (uint64_t i = 0; i < count; i++) v[i] = e.get(vf + i * ts, ts);
      } else {
        const uint64_t off = e.get(vf, inline_bytes);
        if (off + bytes > file_size_) {
          err = "field data outside the file";
          return false;
        }
        std::vector<uint8_t> raw(bytes);
        if (!pread_all(fd_, raw.data(), bytes, off)) {
          err = "cannot read field data";
          return false;
        }
        for (uint64_t i = 0; i < count; i++) v[i] = e.get(raw.data() + i * ts, ts);
      }
      switch (tag) {
        case kWidth: d.width = (uint32_t)v[0]; has_w = true; break;
        case kLength: d.length = (uint32_t)v[0]; has_l = true; break;
        case kBits: d.bits = (uint32_t)v[0]; break;
        case kCompression: d.compression = (uint32_t)v[0]; break;
        case kSpp: d.spp = (uint32_t)v[0]; break;
        case kRowsPerStrip: d.rows_per_strip = (uint32_t)v[0]; break;
        case kPredictor: d.predictor = (uint32_t)v[0]; break;
        case kStripOffsets: d.offsets = v; has_off = true; break;
        case kStripByteCounts: d.counts = v; has_cnt = true; break;
      }
    }
    const int index = (int)dirs_.size();
    auto bad = [&](const std::string& what) {
      err = "directory " + std::to_string(index) + ": " + what;
      return false;
    };
    if (d.tiled) return bad("tiled images are not supported (strips only)");
    if (!has_w || !has_l || !has_off || !has_cnt || d.width == 0 || d.length == 0)
      return bad("missing ImageWidth, ImageLength, StripOffsets or StripByteCounts");
    if (d.spp != 1) return bad("only one sample per pixel is supported");
    if (d.bits != 8 && d.bits != 16) return bad("Only 8-bit or 16-bit TIFF is supported");
    if (d.compression != 1 && d.compression != 5 && d.compression != 8 && d.compression != 32946 &&
        d.compression != 32773)
      return bad("compression " + std::to_string(d.compression) +
                 " is not supported (none, LZW, Deflate, PackBits)");
    if (d.predictor != 1 && d.predictor != 2) return bad("only predictor 1 or 2 is supported");
    const uint64_t rps = std::min<uint64_t>(d.rows_per_strip ? d.rows_per_strip : d.length, d.length);
    const uint64_t nstrips = (d.length + rps - 1) / rps;
    if (d.offsets.size() != nstrips || d.counts.size() != nstrips) return bad("strip tables do not cover the image");
    for (uint64_t s = 0; s < nstrips; s++)
      if (d.offsets[s] + d.counts[s] > file_size_) return bad("strip outside the file");
    d.rows_per_strip = (uint32_t)rps;
    if (!dirs_.empty()) {
      const TiffDir& f = dirs_[0];
      if (d.width != f.width || d.length != f.length || d.bits != f.bits)
        return bad("image size or bit depth differs from the first directory");
    }
    dirs_.push_back(std::move(d));
    const uint8_t* nx = ents.data() + nent * entry_bytes;
    ifd = e.get(nx, inline_bytes);
  }
  if (dirs_.empty()) {
    err = "no image directory";
    return false;
  }
  return true;
}

bool TiffFile::read_image(int i, void* dst, std::string& err) const {
  if (i < 0 || i >= ndirs()) {
    err = "directory index out of range";
    return false;
  }
  const TiffDir& d = dirs_[i];
  const size_t bpp = d.bits / 8, row_bytes = (size_t)d.width * bpp;
  uint8_t* out = static_cast<uint8_t*>(dst);
  std::vector<uint8_t> buf;
  const size_t nstrips = d.offsets.size();
  for (size_t s = 0; s < nstrips; s++) {
    const size_t row0 = s * d.rows_per_strip;
    const size_t rows = std::min<size_t>(d.rows_per_strip, d.length - row0);
    const size_t want = rows * row_bytes;
    uint8_t* o = out + row0 * row_bytes;
    buf.resize(d.counts[s]);
    if (!pread_all(fd_, buf.data(), buf.size(), d.offsets[s])) {
      err = "read error on strip " + std::to_string(s);
      return false;
    }
    bool ok = false;
    switch (d.compression) {
      case 1:
        ok = buf.size() >= want;
        if (ok) std::memcpy(o, buf.data(), want);
        break;
      case 5: ok = tiff_lzw_decode(buf.data(), buf.size(), o, want); break;
      case 8:
      case 32946: ok = tiff_deflate_decode(buf.data(), buf.size(), o, want); break;
      case 32773: ok = tiff_packbits_decode(buf.data(), buf.size(), o, want); break;
    }
    if (!ok) {
      err = "cannot decode strip " + std::to_string(s) + " of directory " + std::to_string(i);
      return false;
    }
    if (bpp == 2 && big_endian_)
      for (size_t k = 0; k < want; k += 2) std::swap(o[k], o[k + 1]);
    if (d.predictor == 2) {
      for (size_t r = 0; r < rows; r++) {
        if (bpp == 1) {
          uint8_t* p = o + r * row_bytes;
          for (size_t x = 1; x < d.width; x++) p[x] = (uint8_t)(p[x] + p[x - 1]);
        } else {
          uint16_t* p = reinterpret_cast<uint16_t*>(o + r * row_bytes);
          for (size_t x = 1; x < d.width; x++) p[x] = (uint16_t)(p[x] + p[x - 1]);
        }
      }
    }
  }
  return true;
}

}  // namespace mc
