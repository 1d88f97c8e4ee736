// Multi-lane stress of the batch runner through the C ABI (include/mc.h):
// movies of three geometries and pixel types, uneven depth and pair
// distance, frames alternately in device memory, pinned host memory and
// pageable host memory, run through mc_batch_run with several lanes and
// several times in a row (plans re-targeted and graphs replayed), each movie
// compared bit for bit with a fresh one-at-a-time plan.  Built and run by
// tests/test_gpu_batch.py, also against an AddressSanitizer build of libmc
// (python -m motioncorr1exp_b200.build --sanitize address).
//
//   batch_stress [lanes] [movies] [rounds]   exit 0 when every result matches
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mc.h"

namespace {

struct Geo {
  int nx, ny, mode;
};
const Geo kGeo[] = {{256, 256, 0}, {300, 290, 0}, {384, 384, 2}};

uint64_t lcg(uint64_t& s) {
  s = s * 6364136223846793005ULL + 1442695040888963407ULL;
  return s >> 33;
}

// frames: a smooth pattern drifting by a whole pixel per frame in x and
// every other frame in y, plus pseudo-random counts
std::vector<unsigned char> make_frames(const Geo& g, int nz, uint64_t seed) {
  const int wl = g.mode == 2 ? 4 : 1;
  std::vector<unsigned char> raw((size_t)nz * g.nx * g.ny * wl);
  uint64_t s = seed;
  for (int f = 0; f < nz; f++)
    for (int y = 0; y < g.ny; y++)
      for (int x = 0; x < g.nx; x++) {
        const int xs = x + f, ys = y + f / 2;
        const int v = ((xs / 7 + ys / 5) % 3) + (int)(lcg(s) % 3);
        const size_t i = ((size_t)f * g.ny + y) * g.nx + x;
        if (wl == 1)
          raw[i] = (unsigned char)v;
        else {
          const float fv = (float)v;
          std::memcpy(&raw[i * 4], &fv, 4);
        }
      }
  return raw;
}

struct Movie {
  int geo, nz;
  mc_params p;
  std::vector<unsigned char> host;
  void* dev = nullptr;
  void* pinned = nullptr;
  int source;  // 0 device, 1 pinned host, 2 pageable host
  int n;
  std::vector<float> ref_image, image;
  std::vector<double> ref_shift, shift;
};

#define CHECK(x)                                                                  \
  do {                                                                            \
    int r_ = (x);                                                                 \
    if (r_ != MC_OK) {                                                            \
      std::fprintf(stderr, "%s:%d %s -> %d %s\n", __FILE__, __LINE__, #x, r_,     \
                   mc_last_error());                                              \
      return 1;                                                                   \
    }                                                                             \
  } while (0)

}  // namespace

int main(int argc, char** argv) {
  const int lanes = argc > 1 ? atoi(argv[1]) : 3;
  const int nmov = argc > 2 ? atoi(argv[2]) : 30;
  const int rounds = argc > 3 ? atoi(argv[3]) : 3;
  std::vector<Movie> mv(nmov);
  uint64_t s = 12345;
  for (int i = 0; i < nmov; i++) {
    Movie& m = mv[i];
    m.geo = (int)(lcg(s) % 3);
    m.nz = 6 + (int)(lcg(s) % 15);
    const Geo& g = kGeo[m.geo];
    mc_default_params(&m.p);
    m.p.CCPeakSearchDim = 64;
    m.p.FrameDistOffset = 1 + (int)(lcg(s) % 3);
    if (m.p.FrameDistOffset >= m.nz / 2) m.p.FrameDistOffset = 1;
    if (lcg(s) % 4 == 0) m.p.kiThresh = 0.3f;
    CHECK(mc_verify_params(&m.p, m.nz));
    m.host = make_frames(g, m.nz, 1000 + i);
    m.source = i % 3;
    if (m.source == 0) {
      if (cudaMalloc(&m.dev, m.host.size()) != cudaSuccess) return 2;
      if (cudaMemcpy(m.dev, m.host.data(), m.host.size(), cudaMemcpyHostToDevice) != cudaSuccess) return 2;
    } else if (m.source == 1) {
      if (cudaMallocHost(&m.pinned, m.host.size()) != cudaSuccess) return 2;
      std::memcpy(m.pinned, m.host.data(), m.host.size());
    }
    m.n = (std::min(g.nx, g.ny) / 2) * 2;
  }
  // one at a time through fresh plans
  for (int i = 0; i < nmov; i++) {
    Movie& m = mv[i];
    const Geo& g = kGeo[m.geo];
    mc_plan* pl = nullptr;
    CHECK(mc_plan_create(&m.p, g.nx, g.ny, m.nz, g.mode, &pl));
    mc_info in{};
    CHECK(mc_plan_info(pl, &in));
    m.n = in.nsam;
    CHECK(mc_plan_load_frames(pl, m.host.data(), 0, in.nframe));
    m.ref_image.assign((size_t)m.n * m.n, 0.f);
    m.ref_shift.assign(2 * (size_t)in.nframe, 0.0);
    CHECK(mc_plan_run(pl, m.ref_image.data()));
    CHECK(mc_plan_get_frame_shifts(pl, m.ref_shift.data()));
    mc_plan_destroy(pl);
  }
  mc_batch* b = nullptr;
  CHECK(mc_batch_create(0, lanes, &b));
  int bad = 0;
  for (int r = 0; r < rounds; r++) {
    std::vector<mc_batch_job> jobs(nmov);
    std::vector<mc_batch_result> res(nmov);
    for (int i = 0; i < nmov; i++) {
      Movie& m = mv[i];
      const Geo& g = kGeo[m.geo];
      m.image.assign((size_t)m.n * m.n, -1.f);
      m.shift.assign(m.ref_shift.size(), -1.0);
      mc_batch_job& j = jobs[i];
      std::memset(&j, 0, sizeof(j));
      j.frames = m.source == 0 ? m.dev : (m.source == 1 ? m.pinned : (const void*)m.host.data());
      j.on_device = m.source == 0;
      j.nx = g.nx;
      j.ny = g.ny;
      j.nz = m.nz;
      j.mode = g.mode;
      j.params = m.p;
      j.image = m.image.data();
      j.frame_shifts = m.shift.data();
    }
    // later rounds run the queue in another order
    if (r % 2 == 1) {
      std::vector<mc_batch_job> rev(jobs.rbegin(), jobs.rend());
      std::vector<mc_batch_result> rres(nmov);
      CHECK(mc_batch_run(b, rev.data(), nmov, rres.data()));
    } else {
      CHECK(mc_batch_run(b, jobs.data(), nmov, res.data()));
    }
    for (int i = 0; i < nmov; i++) {
      const Movie& m = mv[i];
      if (std::memcmp(m.image.data(), m.ref_image.data(), m.image.size() * sizeof(float)) ||
          std::memcmp(m.shift.data(), m.ref_shift.data(), m.shift.size() * sizeof(double))) {
        std::fprintf(stderr, "round %d movie %d (geometry %d, %d frames, source %d) differs\n", r, i, m.geo, m.nz,
                     m.source);
        bad++;
      }
    }
  }
  mc_batch_destroy(b);
  for (auto& m : mv) {
    if (m.dev) cudaFree(m.dev);
    if (m.pinned) cudaFreeHost(m.pinned);
  }
  std::printf("batch stress: %d lanes, %d movies, %d rounds, %d mismatches\n", lanes, nmov, rounds, bad);
  return bad ? 1 : 0;
}
