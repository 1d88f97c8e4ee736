// Minimal strip-TIFF reader for movie stacks: one image per directory,
// one sample per pixel, 8- or 16-bit, strips (no tiles), compression none,
// LZW, Deflate or PackBits, horizontal predictor.  Classic TIFF and BigTIFF,
// either byte order.  It stands in for the libtiff calls of MRCT
// (mrct.cpp:29-152: TIFFOpen, the directory count of fakeReadHeader,
// TIFFReadEncodedStrip per strip) without linking libtiff.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace mc {

struct TiffDir {
  uint32_t width = 0, length = 0;
  uint32_t bits = 1, compression = 1, predictor = 1, spp = 1, rows_per_strip = 0xffffffffu;
  bool tiled = false;
  std::vector<uint64_t> offsets, counts;
};

class TiffFile {
 public:
  TiffFile() = default;
  ~TiffFile();
  TiffFile(const TiffFile&) = delete;
  TiffFile& operator=(const TiffFile&) = delete;

  // Reads the byte-order mark, the magic and the whole directory chain;
  // false with a message when the file is not a TIFF this reader decodes.
  bool open(const char* path, std::string& err);
  int ndirs() const { return (int)dirs_.size(); }
  const TiffDir& dir(int i) const { return dirs_[i]; }
  // Pixels of directory i in host byte order, width*length*bits/8 bytes.
  // Safe to call from several threads at once (positioned reads).
  bool read_image(int i, void* dst, std::string& err) const;

 private:
  int fd_ = -1;
  bool big_endian_ = false;
  uint64_t file_size_ = 0;
  std::vector<TiffDir> dirs_;
};

// Codecs, exposed for the reader's tests through the library: each decodes
// src into exactly `want` bytes of dst and returns false when the stream
// ends early or is malformed.
bool tiff_lzw_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t want);
bool tiff_packbits_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t want);
bool tiff_deflate_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t want);

}  // namespace mc
