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
#include "mc_internal.h"

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
  // single-graph mode (mc_batch_set_graph): the whole batch captured as one
  // CUDA graph on `gst` and launched once; pinned per-movie blocks in `pin`
  bool graph = false;
  cudaStream_t gst = nullptr;
  std::vector<cudaEvent_t> gev;
  unsigned char* pin = nullptr;
  size_t pin_bytes = 0;
  cudaGraphExec_t gexec = nullptr;
  std::vector<unsigned char> gkey;  // the job list the cached graph was captured for
  ~mc_batch() {
    if (gexec) cudaGraphExecDestroy(gexec);
    for (auto e : gev) cudaEventDestroy(e);
    if (gst) cudaStreamDestroy(gst);
    if (pin) cudaFreeHost(pin);
  }
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

int mc_batch_set_graph(mc_batch* b, int on) {
  if (!b) return mc::record_error(MC_E_ARG, "null batch");
  b->graph = on != 0;
  return MC_OK;
}

}  // extern "C"

namespace {

#define BCK(call)                                                                               \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      char m_[256];                                                                             \
      std::snprintf(m_, sizeof(m_), "%s failed: %s", #call, cudaGetErrorString(e_));           \
      return mc::record_error(MC_E_CUDA, m_);                                                   \
    }                                                                                           \
  } while (0)

size_t align64(size_t x) { return (x + 63) / 64 * 64; }

// The whole batch as one CUDA graph: every movie's device-only pipeline
// (forward transforms, pair stage, FP64 solve, sum, C2R, result copies)
// captured in job order, lane l taking jobs l, l + lanes, ... on its own
// plans and running as its own branch of the graph; the graph is launched
// once and the host reads every movie's results after one synchronisation.
// The captured graph is kept and relaunched while the job list is the same.
int run_graph_impl(mc_batch* b, const mc_batch_job* jobs, int njobs, mc_batch_result* results,
                   const std::map<GeoKey, std::pair<int, int>>& need);

// A failure of the batch as a whole (a job the mode cannot take, a capture
// error) is every movie's status, with mc_last_error()'s text.
int run_graph(mc_batch* b, const mc_batch_job* jobs, int njobs, mc_batch_result* results,
              const std::map<GeoKey, std::pair<int, int>>& need) {
  const int rc = run_graph_impl(b, jobs, njobs, results, need);
  if (rc != MC_OK) {
    const std::string text = mc_last_error();
    for (int i = 0; i < njobs; i++)
      if (results[i].status == MC_E_STATE && results[i].lane < 0) {
        results[i].status = rc;
        std::snprintf(results[i].message, sizeof(results[i].message), "%s", text.c_str());
      }
    mc::record_error(rc, text.c_str());
  }
  return rc;
}

int run_graph_impl(mc_batch* b, const mc_batch_job* jobs, int njobs, mc_batch_result* results,
                   const std::map<GeoKey, std::pair<int, int>>& need) {
  const auto t0 = std::chrono::steady_clock::now();
  const int nl = (int)b->lanes.size();
  if (cudaSetDevice(b->device) != cudaSuccess) {
    cudaGetLastError();
    return mc::record_error(MC_E_CUDA, "cudaSetDevice failed");
  }
  for (int i = 0; i < njobs; i++) {
    const mc_batch_job& j = jobs[i];
    if (!j.on_device) return mc::record_error(MC_E_ARG, "graph mode needs the frames in device memory");
    if (j.params.iter != 0 || j.params.refine != 0)
      return mc::record_error(MC_E_ARG, "graph mode runs device-only movies (-itr 0, no refinement)");
    if (j.params.GPUNum != b->device) return mc::record_error(MC_E_ARG, "job GPUNum differs from the runner's GPU");
    if (j.image) {
      cudaPointerAttributes at{};
      if (cudaPointerGetAttributes(&at, j.image) != cudaSuccess ||
          (at.type != cudaMemoryTypeHost && at.type != cudaMemoryTypeDevice)) {
        cudaGetLastError();
        return mc::record_error(MC_E_ARG, "graph mode needs images in pinned host or device memory");
      }
    }
  }
  // plans: lane l, geometry g, capacity of the deepest movie of g
  std::vector<mc_plan*> plan_of(njobs, nullptr);
  for (int i = 0; i < njobs; i++) {
    const mc_batch_job& j = jobs[i];
    Lane& lane = *b->lanes[i % nl];
    const GeoKey key = geo_key(j);
    const auto cap = need.at(key);
    Lane::Entry& e = lane.plans[key];
    if (e.plan && (e.cap_frames < cap.first || e.cap_pairs < cap.second)) {
      mc_plan_destroy(e.plan);
      e.plan = nullptr;
    }
    if (!e.plan) {
      const int rc = mc_plan_create_capacity(&j.params, j.nx, j.ny, j.nz, j.mode, cap.first, cap.second, &e.plan);
      if (rc != MC_OK) {
        e.plan = nullptr;
        return rc;
      }
      e.cap_frames = cap.first;
      e.cap_pairs = cap.second;
    }
    mc_info in{};
    mc_plan_info(e.plan, &in);
    if (in.spectrum_slots)
      return mc::record_error(MC_E_STATE,
                              "graph mode needs every spectrum of a movie in HBM; a plan of this batch holds "
                              "fewer (spectrum slots): run the batch with lanes");
    plan_of[i] = e.plan;
  }
  // pinned per-movie blocks: frame word, pair words, result block
  std::vector<size_t> off_word(njobs), off_pairs(njobs), off_stage(njobs);
  size_t total = 0;
  for (int i = 0; i < njobs; i++) {
    int nf, np;
    job_counts(jobs[i], &nf, &np);
    off_word[i] = total;
    total += 64;
    off_pairs[i] = total;
    total += align64(sizeof(int) * 2 * (size_t)std::max(np, 1));
    off_stage[i] = total;
    total += align64(mc::plan_stage_bytes(plan_of[i]));
  }
  // the job list (and the plans it maps to) the graph is captured for
  std::vector<unsigned char> key(sizeof(mc_batch_job) * njobs + sizeof(mc_plan*) * njobs);
  for (int i = 0; i < njobs; i++) {
    mc_batch_job k = jobs[i];
    k.frame_shifts = nullptr;  // filled on the host after the launch
    std::memcpy(key.data() + sizeof(mc_batch_job) * i, &k, sizeof(k));
  }
  std::memcpy(key.data() + sizeof(mc_batch_job) * njobs, plan_of.data(), sizeof(mc_plan*) * njobs);
  if (b->gexec && (key != b->gkey || total > b->pin_bytes)) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  if (total > b->pin_bytes) {
    if (b->pin) cudaFreeHost(b->pin);
    b->pin = nullptr;
    b->pin_bytes = 0;
    BCK(cudaMallocHost(&b->pin, total));
    b->pin_bytes = total;
  }
  if (!b->gst) BCK(cudaStreamCreateWithFlags(&b->gst, cudaStreamNonBlocking));
  while ((int)b->gev.size() < njobs + 1) {
    cudaEvent_t e;
    BCK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->gev.push_back(e);
  }
  if (!b->gexec) {
    // the words the graph's copies read when it runs
    for (int i = 0; i < njobs; i++) {
      int rc = mc::plan_reframe_host(plan_of[i], &jobs[i].params, jobs[i].nz);
      int nf, np;
      job_counts(jobs[i], &nf, &np);
      if (rc == MC_OK) rc = mc::plan_pair_words(plan_of[i], (int*)(b->pin + off_pairs[i]), std::max(np, 1));
      if (rc != MC_OK) return rc;
      *(const void**)(b->pin + off_word[i]) = jobs[i].frames;
    }
    BCK(cudaStreamBeginCapture(b->gst, cudaStreamCaptureModeThreadLocal));
    int rc = MC_OK;
    cudaError_t ce = cudaEventRecord(b->gev[njobs], b->gst);
    std::vector<cudaEvent_t> last(nl, b->gev[njobs]);
    for (int i = 0; i < njobs && rc == MC_OK && ce == cudaSuccess; i++) {
      mc_plan* pl = plan_of[i];
      rc = mc::plan_reframe_host(pl, &jobs[i].params, jobs[i].nz);
      if (rc != MC_OK) break;
      const cudaStream_t ps = mc::plan_stream(pl);
      ce = cudaStreamWaitEvent(ps, last[i % nl], 0);
      if (ce != cudaSuccess) break;
      rc = mc::plan_enqueue_movie(pl, (const void* const*)(b->pin + off_word[i]), (const int*)(b->pin + off_pairs[i]),
                                  b->pin + off_stage[i], jobs[i].image);
      if (rc != MC_OK) break;
      ce = cudaEventRecord(b->gev[i], ps);
      last[i % nl] = b->gev[i];
    }
    for (int l = 0; l < nl && rc == MC_OK && ce == cudaSuccess; l++) ce = cudaStreamWaitEvent(b->gst, last[l], 0);
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(b->gst, &g);
    if (rc == MC_OK && (ce != cudaSuccess || ee != cudaSuccess || !g)) {
      char m[256];
      std::snprintf(m, sizeof(m), "batch graph capture failed: %s",
                    cudaGetErrorString(ce != cudaSuccess ? ce : ee));
      rc = mc::record_error(MC_E_CUDA, m);
    }
    if (rc == MC_OK) {
      const cudaError_t ie = cudaGraphInstantiate(&b->gexec, g, 0);
      if (ie != cudaSuccess) {
        b->gexec = nullptr;
        char m[256];
        std::snprintf(m, sizeof(m), "batch graph instantiation failed: %s", cudaGetErrorString(ie));
        rc = mc::record_error(MC_E_CUDA, m);
      }
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (rc != MC_OK) return rc;
    b->gkey = key;
  }
  BCK(cudaGraphLaunch(b->gexec, b->gst));
  BCK(cudaStreamSynchronize(b->gst));
  const double t_done = now_ms(t0);
  int first_bad = MC_OK;
  for (int i = 0; i < njobs; i++) {
    mc_batch_result& r = results[i];
    r.lane = i % nl;
    r.start_ms = 0.0;
    mc_plan* pl = plan_of[i];
    int rc = mc::plan_reframe_host(pl, &jobs[i].params, jobs[i].nz);
    if (rc == MC_OK) rc = mc::plan_finish_movie(pl, b->pin + off_stage[i], jobs[i].frames);
    if (rc == MC_OK && jobs[i].frame_shifts) rc = mc_plan_get_frame_shifts(pl, jobs[i].frame_shifts);
    if (rc == MC_OK) {
      mc_info in{};
      mc_plan_info(pl, &in);
      r.nsam = in.nsam;
      r.nframe = in.nframe;
      r.npairs = in.npairs;
    }
    r.gpu_ms = 0.f;
    r.status = rc;
    if (rc != MC_OK) {
      std::snprintf(r.message, sizeof(r.message), "%s", mc_last_error());
      if (first_bad == MC_OK) first_bad = rc;
    }
    r.end_ms = t_done;
  }
  if (first_bad != MC_OK) {
    for (int i = 0; i < njobs; i++)
      if (results[i].status != MC_OK) return mc::record_error(results[i].status, results[i].message);
  }
  return MC_OK;
}

}  // namespace

extern "C" {

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
  if (b->graph && njobs > 0) return run_graph(b, jobs, njobs, results, need);
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
