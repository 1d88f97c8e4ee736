// MRC stack access for the CLI: the 1024-byte header of struct MRCHeader
// (mrcheader.h:3-45), frame n at 1024 + nsymbt + n * nx*ny*wordlength
// (mrc.cpp:151-157), and a mode-2 writer with the header createMRC(float*)
// produces (mrc.cpp:243-274).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>

#pragma pack(push, 1)
struct MrcHeader {
  int32_t nx, ny, nz, mode;
  int32_t nxstart, nystart, nzstart;
  int32_t mx, my, mz;
  float cella[3];
  float cellb[3];
  int32_t mapc, mapr, maps;
  float dmin, dmax, dmean;
  int32_t ispg, nsymbt;
  char extra[100];
  float origin[3];
  char map[4];
  int32_t machst;
  float rms;
  int32_t nlabels;
  char label[10][80];
};
#pragma pack(pop)
static_assert(sizeof(MrcHeader) == 1024, "MRC header must be 1024 bytes");

// MRC::getWordLength (mrc.cpp:99-118)
int mrc_word_length(int mode);

class MrcStack {
 public:
  MrcStack() = default;
  ~MrcStack();
  MrcStack(const MrcStack&) = delete;
  MrcStack& operator=(const MrcStack&) = delete;
  // 1 ok, 0 cannot open, -1 short header (MRC::open, mrc.cpp:29-40)
  int open(const char* path);
  void close();
  const MrcHeader& header() const { return h_; }
  size_t frame_bytes() const;
  // raw bytes of frames [first, first+count) into dst; returns frames read
  int read_frames(void* dst, int first, int count);
  // one frame converted to float (MRC::read2DIm_32bit, mrc.cpp:325-382)
  bool read_frame_float(float* dst, int n);

 private:
  FILE* fp_ = nullptr;
  MrcHeader h_{};
};

// Format detection of isMRC (func.cpp:557-578): 'MAP ' stamp, or a file
// name containing "mrc".
// verb also prints the old-MRC line (isMRC's verb argument).
bool is_mrc(const char* path, bool verb);
bool starts_with_gzip(const char* path);
bool starts_with_tiff(const char* path);

// createMRC(float*) semantics; fills dmin/dmax/dmean; returns false on I/O error.
bool write_mrc_float(const char* path, const float* data, int nx, int ny, int nz, MrcHeader* out_header);

// createMRC(short*) semantics (mrc.cpp:276-307): mode 1, the same geometry
// fields, dmin/dmax/dmean of the shorts; returns false on I/O error.
bool write_mrc_short(const char* path, const int16_t* data, int nx, int ny, int nz);

// Corrected-stack writer: the header a default MRC() object carries
// (mrc.cpp:5-16: mode 2, cellb 90, mapc/mapr/maps 1/2/3, statistics 0) with
// nx, ny, nz set and written by updateHeader (mrc.cpp:237-241); frame n at
// 1024 + n * nx*ny*4 as write2DIm puts it (mrc.cpp:188-194).
class MrcStackWriter {
 public:
  MrcStackWriter() = default;
  ~MrcStackWriter();
  MrcStackWriter(const MrcStackWriter&) = delete;
  MrcStackWriter& operator=(const MrcStackWriter&) = delete;
  bool open(const char* path, int nx, int ny, int nz);
  bool write_frame(const float* data, int n);
  bool close();

 private:
  FILE* fp_ = nullptr;
  int nx_ = 0, ny_ = 0;
};
