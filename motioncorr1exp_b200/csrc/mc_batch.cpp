// Multi-movie batch runner of libmc (mc_batch_* in include/mc.h).
//
// The reference aligns one movie per process (dosefgpu_driftcorr.cpp:121-515).
// Here one runner serves a queue of movies of mixed geometry and depth on one
// GPU: `lanes` host threads, each with its own plans (one per stack
// geometry, created with the capacity of the deepest movie of that geometry
// in the batch and re-targeted per movie with mc_plan_reframe), its own
// stream, and per frame configuration a captured CUDA graph.  Lanes overlap
// one movie's host upload and host-side bookkeeping with the kernels of the
// others, and fill the GPU during each movie's small tail kernels (peak
// search, FP64 solve, C2R).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/mc.h"

namespace mc {
int record_error(int code, const char* text);  // mc_plan.cu: sets mc_last_error()
}

namespace {

// Everything that fixes a plan's buffers and tables.
using GeoKey = std::tuple<int, int, int, int, int, int, int, int, int, int>;

GeoKey geo_key(const mc_batch_job& j) {
  const mc_params& p = j.params;
  int bin_bits;
  std::memcpy(&bin_bits, &p.bin, sizeof(int));
  return GeoKey(j.nx, j.ny, j.mode, p.crop_offsetx, p.crop_offsety, p.crop_nsam, bin_bits, p.CCPeakSearchDim,
                (int)std::lround(p.bfactor * 1000.0f), p.NoisePeakSize);
}

// Aligned frame count and pair count of a job (DFAlign.cu:528-530, mfunc.h:64-84).
void job_counts(const mc_batch_job& j, int* nframe, int* npairs) {
  const int ns = std::max(j.params.nStart, 0), ne = std::min(j.params.nEnd, j.nz - 1);
  const int nf = ne - ns + 1;
  *nframe = nf;
  *npairs = 0;
  if (nf < 2) return;
  int dist = nf / 2 - j.params.FrameDistOffset;
  if (dist <= 0) dist = 1;
  if (dist > nf / 2) dist = nf / 2;
  int np = 0;
  for (int i = 0; i < nf; i++) np += std::max(0, nf - (i + dist));
  *npairs = np;
}

struct Lane {
  struct Entry {
    mc_plan* plan = nullptr;
    int cap_frames = 0, cap_pairs = 0;
  };
  std::map<GeoKey, Entry> plans;
  ~Lane() {
    for (auto& kv : plans) mc_plan_destroy(kv.second.plan);
  }
};

double now_ms(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct mc_batch {
  int device = 0;
  std::vector<std::unique_ptr<Lane>> lanes;
};

extern "C" {

int mc_batch_create(int device, int lanes, mc_batch** out) {
  if (!out || lanes < 1 || lanes > 16) return mc::record_error(MC_E_ARG, "lanes must be in [1, 16]");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
    cudaGetLastError();
    return mc::record_error(MC_E_CUDA, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return mc::record_error(MC_E_ARG, "GPU ID out of range");
  mc_batch* b = new mc_batch();
  b->device = device;
  for (int i = 0; i < lanes; i++) b->lanes.emplace_back(new Lane());
  *out = b;
  return MC_OK;
}

void mc_batch_destroy(mc_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  delete b;
}

size_t mc_batch_device_bytes(const mc_batch* b) {
  if (!b) return 0;
  size_t t = 0;
  for (const auto& l : b->lanes)
    for (const auto& kv : l->plans) {
      mc_info in{};
      if (mc_plan_info(kv.second.plan, &in) == MC_OK) t += in.device_bytes;
    }
  return t;
}

int mc_batch_run(mc_batch* b, const mc_batch_job* jobs, int njobs, mc_batch_result* results) {
  if (!b || (njobs > 0 && (!jobs || !results)) || njobs < 0) return mc::record_error(MC_E_ARG, "null argument");
  // capacity per geometry: the deepest movie of the batch
  std::map<GeoKey, std::pair<int, int>> need;
  for (int i = 0; i < njobs; i++) {
    int nf, np;
    job_counts(jobs[i], &nf, &np);
    auto& c = need[geo_key(jobs[i])];
    c.first = std::max(c.first, nf);
    c.second = std::max(c.second, np);
    results[i] = mc_batch_result{};
    results[i].status = MC_E_STATE;
    results[i].lane = -1;
  }
  const auto t0 = std::chrono::steady_clock::now();
  std::atomic<int> next(0);
  auto work = [&](int li) {
    Lane& lane = *b->lanes[li];
    if (cudaSetDevice(b->device) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= njobs) break;
      const mc_batch_job& j = jobs[i];
      mc_batch_result& r = results[i];
      r.lane = li;
      r.start_ms = now_ms(t0);
      int rc = MC_OK;
      mc_plan* pl = nullptr;
      if (j.params.GPUNum != b->device) rc = mc::record_error(MC_E_ARG, "job GPUNum differs from the runner's GPU");
      if (rc == MC_OK) {
        const GeoKey key = geo_key(j);
        const auto cap = need.at(key);
        Lane::Entry& e = lane.plans[key];
        if (e.plan && (e.cap_frames < cap.first || e.cap_pairs < cap.second)) {
          mc_plan_destroy(e.plan);
          e.plan = nullptr;
        }
        if (!e.plan) {
          rc = mc_plan_create_capacity(&j.params, j.nx, j.ny, j.nz, j.mode, cap.first, cap.second, &e.plan);
          if (rc == MC_OK) {
            e.cap_frames = cap.first;
            e.cap_pairs = cap.second;
          } else {
            e.plan = nullptr;
          }
        } else {
          rc = mc_plan_reframe(e.plan, &j.params, j.nz);
        }
        pl = e.plan;
      }
      if (rc == MC_OK) {
        if (j.on_device) {
          rc = mc_plan_bind_frames_device(pl, j.frames);
          if (rc == MC_OK) rc = mc_plan_run(pl, j.image);
        } else {
          rc = mc_plan_run_host(pl, j.frames, j.image);
        }
      }
      if (rc == MC_OK && j.frame_shifts) rc = mc_plan_get_frame_shifts(pl, j.frame_shifts);
      if (rc == MC_OK) {
        mc_info in{};
        mc_timings tm{};
        mc_plan_info(pl, &in);
        mc_plan_get_timings(pl, &tm);
        r.nsam = in.nsam;
        r.nframe = in.nframe;
        r.npairs = in.npairs;
        r.gpu_ms = tm.total_ms;
      }
      if (pl && j.on_device) mc_plan_bind_frames_device(pl, nullptr);
      r.status = rc;
      if (rc != MC_OK) std::snprintf(r.message, sizeof(r.message), "%s", mc_last_error());
      r.end_ms = now_ms(t0);
    }
  };
  const int nl = std::min((int)b->lanes.size(), std::max(njobs, 1));
  if (nl == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int l = 0; l < nl; l++) th.emplace_back(work, l);
    for (auto& t : th) t.join();
  }
  for (int i = 0; i < njobs; i++)
    if (results[i].status != MC_OK) return mc::record_error(results[i].status, results[i].message);
  return MC_OK;
}

}  // extern "C"
