// Host orchestration and C ABI of libmc (include/mc.h).
//
// One plan = one stack geometry on one GPU.  The whole aligned frame range
// stays resident in HBM: raw frames (file pixel type), their half spectra
// (column-major, see kernels.cuh), the per-pair scratch and the sum buffers.
// Per movie the host only solves the small FP64 least-squares system.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mc.h"
#include "kernels.cuh"
#include "lsq.h"
#include "mc_internal.h"

using mc::cplx;
using mc::FftPlan1D;

namespace {

thread_local std::string g_err;

// Host-side fault injection (mc_debug_fail_alloc): the device or pinned
// allocation that takes this countdown from 1 to 0 fails as if the device
// were out of memory.  0 = off.
std::atomic<int> g_fail_alloc{0};

// Test hook (mc_debug_device_budget): the free device memory plans see when
// they size their spectrum store; 0 = the real figure.
std::atomic<size_t> g_device_budget{0};

bool injected_alloc_failure() {
  int v = g_fail_alloc.load();
  while (v > 0)
    if (g_fail_alloc.compare_exchange_weak(v, v - 1)) return v == 1;
  return false;
}

int set_err(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

}  // namespace

int mc::record_error(int code, const char* text) { return set_err(code, "%s", text); }

namespace {

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return set_err(MC_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                     __LINE__);                                                                    \
  } while (0)

#define CKR(expr)           \
  do {                      \
    int r_ = (expr);        \
    if (r_ != MC_OK) return r_; \
  } while (0)

constexpr double kPi = 3.14159265358979323846;
constexpr int kPairBatch = 512;
constexpr int kPairsPerCta = 32;
// spectrum slots: the fewest a plan works with (two blocks of two frames in
// the pair stage), and the device memory the automatic choice leaves free
// (kernel modules, captured graphs, first-use buffers, the caller's own)
constexpr int kMinSlots = 4;
constexpr size_t kKeepFree = (size_t)256 << 20;

inline long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// ----------------------------------------------------------- FFT planning --
const int kFixedRadices[] = {53, 13, 11, 7, 5, 3};

std::vector<int> factor_radices(int n) {
  std::vector<int> r;
  int m = n;
  for (int p : kFixedRadices)
    while (m % p == 0) {
      r.push_back(p);
      m /= p;
    }
  int twos = 0;
  while (m % 2 == 0) {
    twos++;
    m /= 2;
  }
  // remaining primes -> runtime-radix stages (placed first: no twiddles)
  std::vector<int> generic;
  for (int p = 3; (long long)p * p <= m; p += 2)
    while (m % p == 0) {
      generic.push_back(p);
      m /= p;
    }
  if (m > 1) generic.push_back(m);
  std::vector<int> pw;
  while (twos >= 3) {
    if (twos == 4) {
      pw.push_back(4);
      pw.push_back(4);
      twos = 0;
      break;
    }
    pw.push_back(8);
    twos -= 3;
  }
  if (twos == 2) pw.push_back(4);
  if (twos == 1) pw.push_back(2);
  std::vector<int> out = generic;
  out.insert(out.end(), r.begin(), r.end());
  out.insert(out.end(), pw.begin(), pw.end());
  return out;
}

bool make_plan(int n, FftPlan1D& p) {
  std::vector<int> rad = factor_radices(n);
  if ((int)rad.size() > mc::kMaxStages) return false;
  p.n = n;
  p.nst = (int)rad.size();
  int ns = 1;
  for (int s = 0; s < p.nst; s++) {
    mc::FftStage& st = p.st[s];
    st.R = rad[s];
    st.Ns = ns;
    st.tws = n / (ns * rad[s]);
    st.nsdiv = mc::make_fastdiv((uint32_t)ns);
    st.nqdiv = mc::make_fastdiv((uint32_t)(n / rad[s]));
    ns *= rad[s];
  }
  return ns == n || n == 1;
}

// largest prime factor of n
int max_prime(int n) {
  int best = 1, m = n;
  for (int p = 2; (long long)p * p <= m; p++)
    while (m % p == 0) {
      best = p;
      m /= p;
    }
  return std::max(best, m);
}

double radix_cost(int r) {
  switch (r) {
    case 2: return 2.0;
    case 4: return 2.5;
    case 8: return 3.0;
    case 3: return 3.0;
    case 5: return 4.0;
    case 7: return 5.0;
    case 11: return 7.0;
    case 13: return 8.0;
    default: return (double)r;
  }
}

// Pair-stage schedules by binned side n (mc_schedule_set): the autotuner's
// choices, read when a plan is created.
std::mutex g_sched_mu;
std::map<int, mc_schedule> g_sched;

bool find_schedule(int n, mc_schedule* out) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  auto it = g_sched.find(n);
  if (it == g_sched.end()) return false;
  *out = it->second;
  return true;
}

}  // namespace

// n = P*Q split of the register-codelet column kernel: the split a schedule
// set for n names (mc_schedule_set), else the cheapest by the codelet cost
// model (Q-point FFTs of the P subsequences + 4*box*P outer-sum terms).
// Shared by the plans and mc_pair_window_static, so both run the same kernel.
bool mc::reg_pair_split(int n, int box, int* Pout, int* Qout) {
  int want = 0;
  mc_schedule sc;
  if (find_schedule(n, &sc)) want = sc.pair_q;
  if (want > 1 && n % want == 0 && mc::pair_cols_reg_supported(n / want, want)) {
    *Pout = n / want;
    *Qout = want;
    return true;
  }
  double best = 1e300;
  int P = 0, Q = 0;
  for (int q = 2; q <= n; q++) {
    if (n % q || !mc::pair_cols_reg_supported(n / q, q)) continue;
    std::vector<int> rad = factor_radices(q);
    double c = 0.0;
    for (size_t s = 0; s < rad.size(); s++) c += radix_cost(rad[s]) + (s ? 2.0 : 0.0);
    const double cost = (double)n * c + 4.0 * box * (n / q);
    if (cost < best) {
      best = cost;
      P = n / q;
      Q = q;
    }
  }
  if (!P) return false;
  *Pout = P;
  *Qout = Q;
  return true;
}

namespace {

// n = P*Q for the pruned inverse: Q-point FFTs + P-term output sums.
void choose_prune(int n, int box, int& P, int& Q) {
  double best = 1e300;
  if (mc::reg_pair_split(n, box, &P, &Q)) return;
  // otherwise the shared-memory kernel
  P = n;
  Q = 1;
  for (int q = 1; q <= n; q++) {
    if (n % q) continue;
    const int p = n / q;
    if (mc::pair_cols_smem(n, p, q, box) + 16 > 227 * 1024) continue;  // must fit shared memory
    if (q > 1 && max_prime(q) > 13) continue;
    double c = 0.0;
    if (q > 1) {
      std::vector<int> rad = factor_radices(q);
      for (size_t s = 0; s < rad.size(); s++) c += radix_cost(rad[s]) + (s ? 2.0 : 0.0);
    }
    const double cost = (double)n * c + 4.0 * box * p;
    if (cost < best) {
      best = cost;
      P = p;
      Q = q;
    }
  }
}

std::vector<float2> twiddles(int n, int sign) {
  std::vector<float2> t(n);
  for (int m = 0; m < n; m++) {
    const double a = sign * 2.0 * kPi * (double)m / (double)n;
    t[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  return t;
}

int verify_crop_size(int nx, int ny, int offx, int offy, int nsamout, float fb) {
  if (offx < 0 || offx >= nx || offy < 0 || offy >= ny || fb <= 0) return 0;
  if (nsamout <= 0) nsamout = std::min(nx - offx, ny - offy);
  if (nx - offx < nsamout) nsamout = nx - offx;
  if (ny - offy < nsamout) nsamout = ny - offy;
  if (std::fabs(fb - 1.0) < 0.0001) nsamout = nsamout / 2 * 2;
  else if (std::fabs(fb - 2.0) < 0.0001) nsamout = nsamout / 4 * 4;
  else nsamout = nsamout / 2 * 2;
  return nsamout;
}

int word_length(int mode) {
  switch (mode) {
    case 0: return 1;
    case 1: return 2;
    case 2: return 4;
    case 6: return 2;
    case MC_MODE_U8: return 1;
    case MC_MODE_F16: return 2;
    default: return 0;
  }
}

}  // namespace

// ================================================================= plan ==
struct mc_plan {
  mc_params p{};
  int nx = 0, ny = 0, nz = 0, mode = 0, wl = 0;
  int nstart = 0, nend = 0, nframe = 0;
  int cap_frames = 0, cap_pairs = 0;  // buffer capacities (mc_plan_reframe stays within them)
  int ppc = 32;                       // pairs per CTA of the pair column stage
  int nu = 0, n = 0, H = 0, ldn = 0, ldu = 0, ldt2 = 0;
  int box = 0, ystart = 0, P = 1, Q = 1;
  bool two_sets = false;
  float binf = 1.f;
  size_t frame_bytes = 0;
  long long fstride = 0;  // complex elements per stored spectrum
  size_t dev_bytes = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st_copy = nullptr;          // upload stream of mc_plan_run_host
  std::vector<cudaEvent_t> chunk_ev;       // one per uploaded chunk
  cudaEvent_t start_ev = nullptr;
  int device = 0;
  mc_log_fn logfn = nullptr;
  void* loguser = nullptr;

  FftPlan1D plan_nu{}, plan_n{}, plan_q{};

  // device memory
  void* d_frames = nullptr;
  int* d_count = nullptr;  // exact count sum (allocated on first use)
  float2* d_ql = nullptr;  // quick-look: side-400 spectrum + C2R scratch (first use)
  float* d_qlimg = nullptr;
  double* d_fsc = nullptr;  // FSC: per-column shell tables + the reduced table (first use)
  // -scx/-scy stretch (mc_plan_set_stretch): row/column source maps, one
  // stretched raw frame, and the references gathered through the same maps
  bool stretch = false;
  int *d_rmap = nullptr, *d_cmap = nullptr;
  void* d_sframe = nullptr;
  float *d_dark_s = nullptr, *d_dark2_s = nullptr, *d_norm_s = nullptr, *d_norm2_s = nullptr;
  const void* frames_src = nullptr;  // bound caller device frames (mc_plan_bind_frames_device) or null
  float *d_dark = nullptr, *d_dark2 = nullptr, *d_norm = nullptr, *d_norm2 = nullptr;
  float2 *d_specA = nullptr, *d_specB = nullptr, *d_T = nullptr;
  // spectrum slots: 0 = every frame position keeps its spectrum in HBM;
  // otherwise the store holds `slots` spectra and a stage that needs one it
  // gave up runs that frame's forward transform again (least recently used
  // slot first)
  int slots = 0;
  std::vector<int> slot_frame;     // frame position held by each slot, -1 none
  std::vector<int> frame_slot;     // slot holding each frame position, -1 none
  std::vector<long long> slot_use;  // last use of each slot (0 = empty)
  long long slot_clock = 0, recomputes = 0;
  float* d_boxes_all = nullptr;    // slot mode: pair windows gathered in list order
  float2 *d_tw_nu = nullptr, *d_tw_n = nullptr, *d_twQ = nullptr, *d_twO = nullptr, *d_cs = nullptr;
  float2* d_twN = nullptr;  // length-n outer table of the generic pair kernel (large P x box)
  double* d_w16 = nullptr;
  int2* d_pairs = nullptr;
  float2* d_G = nullptr;
  float* d_boxes = nullptr;
  float *d_pshift = nullptr, *d_pcc = nullptr;
  int* d_ppeak = nullptr;
  float2 *d_sum = nullptr, *d_T2 = nullptr, *d_ey = nullptr;
  float2* d_sumacc = nullptr;  // sum spectrum of the split image sum (two-level n)
  float* d_image = nullptr;
  int *d_sumframes = nullptr, *d_apply = nullptr;
  double2* d_sumshift = nullptr;
  double* d_opart = nullptr;  // objective partials [H][nframe][5] + [H]
  double* d_oout = nullptr;   // objective totals [nframe][5] + J

  // device-only movie pipeline (forward -> pairs -> device solve -> sum)
  int2* d_pairs_main = nullptr;  // the plan's pair list, uploaded once
  double *d_M = nullptr, *d_rhs = nullptr, *d_work = nullptr, *d_ki1 = nullptr, *d_ki2 = nullptr;
  double *d_dshift = nullptr, *d_dfshift = nullptr;
  int *d_mask = nullptr, *d_order = nullptr, *d_uf = nullptr, *d_kept = nullptr, *d_nkept = nullptr;
  int* d_status = nullptr;
  unsigned char* h_stage = nullptr;  // pinned copies of the per-movie results
  const void** d_src_slot = nullptr;  // device word: base of the run's frames (read by the forward kernels)
  size_t st_dc = 0, st_pshift = 0, st_pcc = 0, st_ppeak = 0, st_ki1 = 0, st_kept = 0, st_nkept = 0, st_ki2 = 0,
         st_work = 0, st_status = 0, st_slot = 0, st_bytes = 0;
  // captured movie graphs, one per frame configuration (frame range, sum
  // range, pair distance, threshold, reference frame) the plan has run
  struct GraphEntry {
    std::vector<long long> key;
    cudaGraphExec_t exec = nullptr;
    double kbytes[MC_KERNEL_KINDS] = {};
    long long kcount[MC_KERNEL_KINDS] = {};
  };
  std::vector<GraphEntry> graphs;
  bool graph_failed = false;
  bool capturing = false;
  // forward transforms of independent frames on `nfs` forked streams
  // (parallel branches in a captured movie; 4 unless a schedule sets it), so
  // one frame's last partial wave of CTAs overlaps the next frames' work;
  // the radix-53 pairing of the forward row / column passes (0 built-in)
  static constexpr int kMaxForwardStreams = 8;
  int nfs = 4;
  int fwd_rows_pairing = 0, fwd_cols_pairing = 0;
  cudaStream_t fst[kMaxForwardStreams] = {};
  cudaEvent_t fev[kMaxForwardStreams + 1] = {};
  int maxp = 0;
  std::vector<void*> allocs;

  // state
  bool loaded_all = false, have_forward = false, have_pairs = false, have_solve = false, have_iter = false;
  bool have_sum = false;  // sum_shift / sum_first / sum_last belong to the current shifts
  std::vector<char> loaded;

  // results
  std::vector<mc::PairIJ> pairs;
  std::vector<float> pshift, pcc;
  std::vector<int> ppeak;
  std::vector<float> frame_mean;
  std::vector<double> ki1, ki2;
  std::vector<int> good;
  std::vector<cplx> shift;        // per step (nframe-1)
  std::vector<cplx> frame_shift;  // cumulative (nframe)
  std::vector<cplx> sum_shift;
  int sum_first = 0, sum_last = -1;
  mc_timings tm{};
  cudaEvent_t ev[8]{};

  // per-kernel accounting: launches and algorithmic bytes always, device
  // time (one event pair per launch) when profiling is on
  bool profiling = false;
  std::vector<cudaEvent_t> kpool;
  struct KRec {
    int kind, e0, e1;
  };
  std::vector<KRec> krec;
  int kused = 0;
  double kbytes[MC_KERNEL_KINDS] = {};
  double kms[MC_KERNEL_KINDS] = {};
  long long kcount[MC_KERNEL_KINDS] = {};

  int kevent(cudaEvent_t* e) {
    if (kused == (int)kpool.size()) {
      cudaEvent_t x;
      CK(cudaEventCreate(&x));
      kpool.push_back(x);
    }
    *e = kpool[kused++];
    return MC_OK;
  }
  double graph_kbytes[MC_KERNEL_KINDS] = {};
  long long graph_kcount[MC_KERNEL_KINDS] = {};
  int kstart(int kind, int* slot) {
    *slot = -1;
    if (!profiling || capturing) return MC_OK;
    cudaEvent_t e;
    CKR(kevent(&e));
    CK(cudaEventRecord(e, st));
    krec.push_back({kind, kused - 1, -1});
    *slot = (int)krec.size() - 1;
    return MC_OK;
  }
  int kstop(int kind, int slot, double bytes, int nk = 1) {
    if (capturing) {  // counted once per graph replay instead
      graph_kcount[kind] += nk;
      graph_kbytes[kind] += bytes;
      return MC_OK;
    }
    kcount[kind] += nk;
    kbytes[kind] += bytes;
    if (slot < 0) return MC_OK;
    cudaEvent_t e;
    CKR(kevent(&e));
    CK(cudaEventRecord(e, st));
    krec[slot].e1 = kused - 1;
    return MC_OK;
  }
  // after a stream synchronisation: fold the recorded launches into kms
  int collect() {
    for (const KRec& r : krec) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, kpool[r.e0], kpool[r.e1]));
      kms[r.kind] += ms;
    }
    krec.clear();
    kused = 0;
    return MC_OK;
  }

  void log(const char* fmt, ...) {
    if (!logfn) return;
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    logfn(buf, loguser);
  }

  template <typename T>
  int alloc(T** ptr, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (injected_alloc_failure())
      return set_err(MC_E_NOMEM, "cudaMalloc(%zu bytes) failed: injected failure (mc_debug_fail_alloc)", bytes);
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_err(MC_E_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    allocs.push_back(q);
    dev_bytes += bytes;
    *ptr = (T*)q;
    return MC_OK;
  }

  ~mc_plan() {
    if (device >= 0) cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    for (void* q : allocs) cudaFree(q);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& s : fst)
      if (s) cudaStreamDestroy(s);
    for (auto& e : fev)
      if (e) cudaEventDestroy(e);
    if (h_stage) cudaFreeHost(h_stage);
    for (auto& e : kpool) cudaEventDestroy(e);
    for (auto& e : chunk_ev) cudaEventDestroy(e);
    if (start_ev) cudaEventDestroy(start_ev);
    if (st_copy) {
      cudaStreamSynchronize(st_copy);
      cudaStreamDestroy(st_copy);
    }
    if (st) cudaStreamDestroy(st);
  }
};

// Forward transforms of every frame position into its own spectrum, or of the
// listed (frame, slot) jobs (defined with the forward stage below).
static int enqueue_forward(mc_plan* pl, const std::vector<cudaEvent_t>* waits, int chunk,
                           const std::vector<std::pair<int, int>>* only = nullptr);

namespace {

// launch `call` (a stage of nk kernels) as kernel kind `kind`, moving `bytes`
// algorithmic bytes; the stage is timed once and its nk launches counted
#define LAUNCH_N(pl, kind, bytes, nk, call)         \
  do {                                              \
    int slot_;                                      \
    CKR((pl)->kstart((kind), &slot_));              \
    CK(call);                                       \
    CKR((pl)->kstop((kind), slot_, (bytes), (nk))); \
  } while (0)
#define LAUNCH(pl, kind, bytes, call) LAUNCH_N(pl, kind, bytes, 1, call)

template <typename T>
int upload(mc_plan* pl, T* dst, const std::vector<T>& src) {
  CK(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, pl->st));
  return MC_OK;
}

float2* specA_at(mc_plan* pl, int f) { return pl->d_specA + (long long)f * pl->fstride; }
float2* specB_at(mc_plan* pl, int f) { return pl->d_specB + (long long)f * pl->fstride; }

// Slot mode: forget every held spectrum (new frames, references or range).
void clear_slots(mc_plan* pl) {
  if (!pl->slots) return;
  pl->slot_frame.assign(pl->slots, -1);
  pl->slot_use.assign(pl->slots, 0);
  pl->frame_slot.assign(pl->cap_frames, -1);
}

// The spectra of `frames` (frame positions, at most `slots` distinct ones)
// in the store: `where` receives the spectrum index of each listed frame.
// With every spectrum resident that is the frame position itself; in slot
// mode frames not held are transformed again into the least recently used
// slots that no listed frame occupies, on the plan stream, after the work
// already queued there (which may still read the slots given up).  The
// forward stage's own pass (`first_pass`) is not counted as recomputation.
int hold_spectra(mc_plan* pl, const std::vector<int>& frames, std::vector<int>& where, bool first_pass = false) {
  where = frames;
  if (!pl->slots) return MC_OK;
  std::vector<char> keep(pl->slots, 0);
  for (int f : frames)
    if (pl->frame_slot[f] >= 0) keep[pl->frame_slot[f]] = 1;
  std::vector<std::pair<int, int>> jobs;
  for (int f : frames) {
    int& fs = pl->frame_slot[f];
    if (fs < 0) {
      int best = -1;
      for (int s = 0; s < pl->slots; s++)
        if (!keep[s] && (best < 0 || pl->slot_use[s] < pl->slot_use[best])) best = s;
      if (best < 0) return set_err(MC_E_STATE, "more spectra asked at once than the plan's %d slots", pl->slots);
      if (pl->slot_frame[best] >= 0) pl->frame_slot[pl->slot_frame[best]] = -1;
      pl->slot_frame[best] = f;
      fs = best;
      keep[best] = 1;
      jobs.push_back({f, best});
    }
    pl->slot_use[fs] = ++pl->slot_clock;
  }
  if (!jobs.empty()) {
    CKR(enqueue_forward(pl, nullptr, 1, &jobs));
    if (!first_pass) pl->recomputes += (long long)jobs.size();
  }
  for (size_t i = 0; i < frames.size(); i++) where[i] = pl->frame_slot[frames[i]];
  return MC_OK;
}

// pair stage over an explicit list: (a-frame, b-frame) into a/b spectrum sets
// Launches the pair kernels for `list`, whose device copy is d_list; results
// land in d_pshift / d_pcc / d_ppeak.  No host synchronisation.
int enqueue_pair_stage(mc_plan* pl, const float2* specA, long long strideA, const float2* specB, long long strideB,
                       const std::vector<mc::PairIJ>& list, const int2* d_list) {
  const int np = (int)list.size();
  if (np > pl->maxp) return set_err(MC_E_STATE, "pair list larger than the plan's capacity");
  const float mbf = (float)(-0.5 * (double)pl->p.bfactor / pl->n / pl->n);
  for (int p0 = 0; p0 < np; p0 += kPairBatch) {
    const int nb = std::min(kPairBatch, np - p0);
    mc::PairColsArgs a{};
    a.specA = specA;
    a.strideA = strideA;
    a.specB = specB;
    a.strideB = strideB;
    a.pairs = d_list + p0;
    a.npairs = nb;
    a.pairs_per_cta = pl->ppc;
    a.n = pl->n;
    a.ldn = pl->ldn;
    a.H = pl->H;
    a.mbf = mbf;
    a.inv_size = (float)(1.0 / ((double)(pl->n / 2 + 1) * pl->n));
    a.P = pl->P;
    a.Q = pl->Q;
    a.qplan = pl->plan_q;
    a.twQ = pl->d_twQ;
    a.twO = pl->d_twO;
    a.twN = pl->d_twN;
    a.box = pl->box;
    a.ystart = pl->ystart;
    a.G = pl->d_G;
    // algorithmic bytes: every distinct spectrum the batch touches read once,
    // the column-stage output written once
    // (a shared spectrum set counts once: A and B are the same buffers)
    const bool one_set = specA == specB && strideA == strideB;
    std::vector<char> seenA(pl->nframe + 1, 0), seenB(pl->nframe + 1, 0);
    long long nspec = 0;
    for (int i = p0; i < p0 + nb; i++) {
      const int fa = strideA ? list[i].first : pl->nframe, fb = list[i].second;
      if (!seenA[fa]) {
        seenA[fa] = 1;
        nspec++;
      }
      char& sb = one_set ? seenA[fb] : seenB[fb];
      if (!sb) {
        sb = 1;
        nspec++;
      }
    }
    const double gbytes = (double)nb * pl->H * pl->box * sizeof(float2);
    const double cbytes = (double)nspec * pl->H * pl->n * sizeof(float2) + gbytes;
    LAUNCH(pl, MC_K_PAIR_COLS, cbytes, mc::launch_pair_cols(a, pl->st));
    mc::PairRowsArgs r{};
    r.G = pl->d_G;
    r.npairs = nb;
    r.H = pl->H;
    r.box = pl->box;
    r.cs = pl->d_cs;
    r.boxes = pl->d_boxes + (long long)p0 * pl->box * pl->box;
    r.twO = pl->d_twO;
    r.P = pl->P;
    r.Q = pl->Q;
    r.ystart = pl->ystart;
    LAUNCH(pl, MC_K_PAIR_ROWS,
           gbytes + (double)pl->H * pl->box * sizeof(float2) + (double)nb * pl->box * pl->box * sizeof(float),
           mc::launch_pair_rows(r, pl->st));
  }
  mc::PeakArgs k{};
  k.boxes = pl->d_boxes;
  k.npairs = np;
  k.box = pl->box;
  k.n = pl->n;
  k.nps = pl->p.NoisePeakSize;
  k.w16 = pl->d_w16;
  k.shift = pl->d_pshift;
  k.cc = pl->d_pcc;
  k.peak = pl->d_ppeak;
  LAUNCH(pl, MC_K_PEAK, (double)np * pl->box * pl->box * sizeof(float) + (double)np * 5 * sizeof(float),
         mc::launch_peak(k, pl->st));
  return MC_OK;
}

// pair stage over an explicit list of spectrum indices, synchronous,
// results to the host
int run_pair_list_held(mc_plan* pl, const float2* specA, long long strideA, const float2* specB, long long strideB,
                       const std::vector<mc::PairIJ>& list, std::vector<float>& shift, std::vector<float>& cc,
                       std::vector<int>& peak) {
  const int np = (int)list.size();
  shift.assign(2 * (size_t)np, 0.f);
  cc.assign(np, 0.f);
  peak.assign(2 * (size_t)np, 0);
  std::vector<int2> pr(np);
  for (int i = 0; i < np; i++) pr[i] = make_int2(list[i].first, list[i].second);
  if (np > pl->maxp) return set_err(MC_E_STATE, "pair list larger than the plan's capacity");
  CK(cudaMemcpyAsync(pl->d_pairs, pr.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, pl->st));
  CKR(enqueue_pair_stage(pl, specA, strideA, specB, strideB, list, pl->d_pairs));
  CK(cudaMemcpyAsync(shift.data(), pl->d_pshift, sizeof(float) * 2 * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(cc.data(), pl->d_pcc, sizeof(float) * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(peak.data(), pl->d_ppeak, sizeof(int) * 2 * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  return pl->collect();
}

// Pair stage over a list of frame positions (first = a frame of set A, or
// any index when set A is the sum spectrum, strideA = 0), synchronous,
// results to the host and the windows to d_boxes in list order.  In slot
// mode the list runs in groups whose frames the slots hold at once: against
// the sum, `slots` frames per group; frame against frame, the frames are cut
// into blocks of slots/2 and each group is the pairs between two blocks (or
// within one), so a block is transformed once per block it meets.  Every
// pair is computed by the same kernels as in the resident plan.
int run_pair_list(mc_plan* pl, const float2* specA, long long strideA, const float2* specB, long long strideB,
                  const std::vector<mc::PairIJ>& list, std::vector<float>& shift, std::vector<float>& cc,
                  std::vector<int>& peak) {
  if (!pl->slots) return run_pair_list_held(pl, specA, strideA, specB, strideB, list, shift, cc, peak);
  const int np = (int)list.size();
  const bool vs_sum = strideA == 0;
  shift.assign(2 * (size_t)np, 0.f);
  cc.assign(np, 0.f);
  peak.assign(2 * (size_t)np, 0);
  const size_t box2 = (size_t)pl->box * pl->box;
  if (!pl->d_boxes_all) CKR(pl->alloc(&pl->d_boxes_all, sizeof(float) * box2 * pl->maxp));
  // groups of list positions, keyed by the frame blocks they touch
  std::map<std::pair<int, int>, std::vector<int>> groups;
  const int blk = vs_sum ? pl->slots : pl->slots / 2;
  for (int i = 0; i < np; i++) {
    const int bj = list[i].second / blk;
    const int bi = vs_sum ? bj : list[i].first / blk;
    groups[{std::min(bi, bj), std::max(bi, bj)}].push_back(i);
  }
  // against the sum, the last frames first: they are the ones the sum left held
  std::vector<const std::vector<int>*> order;
  for (auto& g : groups) order.push_back(&g.second);
  if (vs_sum) std::reverse(order.begin(), order.end());
  for (const std::vector<int>* g : order) {
    std::vector<int> fr;
    for (int i : *g) {
      if (!vs_sum) fr.push_back(list[i].first);
      fr.push_back(list[i].second);
    }
    std::sort(fr.begin(), fr.end());
    fr.erase(std::unique(fr.begin(), fr.end()), fr.end());
    std::vector<int> where;
    CKR(hold_spectra(pl, fr, where));
    std::vector<int> slot_of(pl->nframe, -1);
    for (size_t k = 0; k < fr.size(); k++) slot_of[fr[k]] = where[k];
    std::vector<mc::PairIJ> sub;
    for (int i : *g) sub.push_back({vs_sum ? list[i].first : slot_of[list[i].first], slot_of[list[i].second]});
    std::vector<float> s, c;
    std::vector<int> p;
    CKR(run_pair_list_held(pl, specA, strideA, specB, strideB, sub, s, c, p));
    for (size_t r = 0; r < g->size(); r++) {
      const int i = (*g)[r];
      shift[2 * i] = s[2 * r];
      shift[2 * i + 1] = s[2 * r + 1];
      cc[i] = c[r];
      peak[2 * i] = p[2 * r];
      peak[2 * i + 1] = p[2 * r + 1];
      CK(cudaMemcpyAsync(pl->d_boxes_all + (size_t)i * box2, pl->d_boxes + r * box2, sizeof(float) * box2,
                         cudaMemcpyDeviceToDevice, pl->st));
    }
  }
  CK(cudaMemcpyAsync(pl->d_boxes, pl->d_boxes_all, sizeof(float) * box2 * np, cudaMemcpyDeviceToDevice, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  return MC_OK;
}

// sum of phase-shifted frames of set A; mode 0 -> d_sum spectrum, mode 1 -> image
int run_shift_sum_held(mc_plan* pl, const std::vector<int>& frames, const std::vector<cplx>& shifts,
                       const std::vector<int>& apply, int mode, int accumulate = 0) {
  const int ns = (int)frames.size();
  std::vector<double2> sh(ns);
  for (int i = 0; i < ns; i++) sh[i] = make_double2(shifts[i].real(), shifts[i].imag());
  CK(cudaMemcpyAsync(pl->d_sumframes, frames.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, pl->st));
  CK(cudaMemcpyAsync(pl->d_apply, apply.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, pl->st));
  CK(cudaMemcpyAsync(pl->d_sumshift, sh.data(), sizeof(double2) * ns, cudaMemcpyHostToDevice, pl->st));
  mc::ShiftSumArgs a{};
  a.spec = pl->d_specA;
  a.stride = pl->fstride;
  a.frames = pl->d_sumframes;
  a.shifts = pl->d_sumshift;
  a.apply = pl->d_apply;
  a.nsum = ns;
  a.n = pl->n;
  a.ldn = pl->ldn;
  a.H = pl->H;
  a.mode = mode;
  a.plan = pl->plan_n;
  a.tw = pl->d_tw_n;
  a.acc = pl->d_sumacc;
  a.accumulate = accumulate;
  if (mode == 0) {
    a.out = pl->d_sum;
    a.ld_out = pl->ldn;
  } else {
    a.out = pl->d_T2;
    a.ld_out = pl->ldt2;
  }
  const double spec_bytes = (double)pl->H * pl->n * sizeof(float2);
  LAUNCH_N(pl, MC_K_SHIFT_SUM, (double)ns * spec_bytes + spec_bytes, mc::shift_sum_kernels(a),
           mc::launch_shift_sum(a, pl->d_ey, pl->st));
  if (mode == 1) {
    mc::C2rRowsArgs c{};
    c.t2 = pl->d_T2;
    c.ld_t2 = pl->ldt2;
    c.n = pl->n;
    c.H = pl->H;
    c.scale = (float)(1.0 / ((double)pl->n * pl->n));
    c.image = pl->d_image;
    c.plan = pl->plan_n;
    c.tw = pl->d_tw_n;
    LAUNCH(pl, MC_K_C2R_ROWS, spec_bytes + (double)pl->n * pl->n * sizeof(float), mc::launch_c2r_rows(c, pl->st));
  }
  return MC_OK;
}


// The sum of phase-shifted frames (frame positions) as run_shift_sum_held.
// In slot mode the frames are summed `slots` at a time into d_sum, each
// chunk adding onto the last in frame order, so the sum spectrum is the
// resident plan's bit for bit; mode 1 then transforms d_sum as the one
// unshifted term of a sum (0 + S is S exactly).  Leaves the ramps of the
// last chunk in d_ey.
int run_shift_sum(mc_plan* pl, const std::vector<int>& frames, const std::vector<cplx>& shifts,
                  const std::vector<int>& apply, int mode) {
  if (!pl->slots) return run_shift_sum_held(pl, frames, shifts, apply, mode);
  const int ns = (int)frames.size();
  for (int c0 = 0; c0 < ns; c0 += pl->slots) {
    const int cnt = std::min(pl->slots, ns - c0);
    const std::vector<int> fr(frames.begin() + c0, frames.begin() + c0 + cnt);
    std::vector<int> where;
    CKR(hold_spectra(pl, fr, where));
    CKR(run_shift_sum_held(pl, where, std::vector<cplx>(shifts.begin() + c0, shifts.begin() + c0 + cnt),
                           std::vector<int>(apply.begin() + c0, apply.begin() + c0 + cnt), 0, c0 > 0 ? 1 : 0));
  }
  if (mode == 0) return MC_OK;
  mc::ShiftSumArgs a{};
  const std::vector<int> zero{0};
  const std::vector<double2> none{make_double2(0.0, 0.0)};
  CK(cudaMemcpyAsync(pl->d_sumframes, zero.data(), sizeof(int), cudaMemcpyHostToDevice, pl->st));
  CK(cudaMemcpyAsync(pl->d_apply, zero.data(), sizeof(int), cudaMemcpyHostToDevice, pl->st));
  CK(cudaMemcpyAsync(pl->d_sumshift, none.data(), sizeof(double2), cudaMemcpyHostToDevice, pl->st));
  a.spec = pl->d_sum;
  a.stride = 0;
  a.frames = pl->d_sumframes;
  a.shifts = pl->d_sumshift;
  a.apply = pl->d_apply;
  a.nsum = 1;
  a.n = pl->n;
  a.ldn = pl->ldn;
  a.H = pl->H;
  a.mode = 1;
  a.plan = pl->plan_n;
  a.tw = pl->d_tw_n;
  a.acc = pl->d_sumacc;
  a.out = pl->d_T2;
  a.ld_out = pl->ldt2;
  const double spec_bytes = (double)pl->H * pl->n * sizeof(float2);
  LAUNCH_N(pl, MC_K_SHIFT_SUM, 2 * spec_bytes, mc::shift_sum_kernels(a), mc::launch_shift_sum(a, pl->d_ey, pl->st));
  mc::C2rRowsArgs c{};
  c.t2 = pl->d_T2;
  c.ld_t2 = pl->ldt2;
  c.n = pl->n;
  c.H = pl->H;
  c.scale = (float)(1.0 / ((double)pl->n * pl->n));
  c.image = pl->d_image;
  c.plan = pl->plan_n;
  c.tw = pl->d_tw_n;
  LAUNCH(pl, MC_K_C2R_ROWS, spec_bytes + (double)pl->n * pl->n * sizeof(float), mc::launch_c2r_rows(c, pl->st));
  return MC_OK;
}
}  // namespace

// ================================================================== C ABI ==
extern "C" {

int mc_version(void) { return MC_VERSION; }

const char* mc_strerror(int code) {
  switch (code) {
    case MC_OK: return "ok";
    case MC_E_ARG: return "invalid argument";
    case MC_E_CUDA: return "CUDA error";
    case MC_E_NOMEM: return "out of memory";
    case MC_E_SIZE: return "unsupported size";
    case MC_E_STATE: return "call out of order";
    case MC_E_NUMERIC: return "singular least-squares system";
    case MC_E_IO: return "stack file error";
    default: return "unknown error";
  }
}

const char* mc_last_error(void) { return g_err.c_str(); }

void mc_debug_fail_alloc(int nth) { g_fail_alloc.store(nth > 0 ? nth : 0); }

void mc_debug_device_budget(size_t bytes) { g_device_budget.store(bytes); }

void mc_default_params(mc_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->bin = 1.0f;
  p->bfactor = 150.f;
  p->CCPeakSearchDim = 96;
  p->FrameDistOffset = 2;
  p->NoisePeakSize = 0;
  p->kiThresh = 1.0f;
  p->bAlignToMid = 1;
  p->iter = 0;
  p->iterthres = 0.f;
  p->refine = 0;
}

int mc_verify_params(mc_params* p, int nz) {
  if (!p) return set_err(MC_E_ARG, "null params");
  if (nz <= 1) return set_err(MC_E_ARG, "Not a stack or wrong file. Abort");
  if (p->nStart < 0) p->nStart = 0;
  if (p->nEnd >= nz) p->nEnd = nz - 1;
  if (p->nEnd <= p->nStart) p->nEnd = nz - 1;
  if (p->nStartSum < p->nStart) p->nStartSum = p->nStart;
  if (p->nEndSum > p->nEnd) p->nEndSum = p->nEnd;
  if (p->nEndSum <= p->nStartSum) p->nEndSum = p->nEnd;
  if (p->FrameDistOffset >= nz / 2 || p->FrameDistOffset < 0)
    return set_err(MC_E_ARG, "Frame distance offset is too big or less than 0. Abort");
  return MC_OK;
}

void* mc_plan_stream(mc_plan* pl) { return pl ? (void*)pl->st : nullptr; }

void mc_plan_set_log(mc_plan* pl, mc_log_fn fn, void* user) {
  if (!pl) return;
  pl->logfn = fn;
  pl->loguser = user;
}

void mc_plan_destroy(mc_plan* pl) { delete pl; }

}  // extern "C"

// Frame range and pair list of the run (DFAlign.cu:528-530, mfunc.h:64-84);
// the buffers were sized for cap_frames / cap_pairs.
static int configure_frames(mc_plan* pl, const mc_params& q, int nz, bool upload_pairs = true) {
  mc_params& p = pl->p;
  p.nStart = q.nStart;
  p.nEnd = q.nEnd;
  p.nStartSum = q.nStartSum;
  p.nEndSum = q.nEndSum;
  p.FrameDistOffset = q.FrameDistOffset;
  p.kiThresh = q.kiThresh;
  p.bAlignToMid = q.bAlignToMid;
  pl->nz = nz;
  pl->nstart = std::max(p.nStart, 0);
  pl->nend = std::min(p.nEnd, nz - 1);
  pl->nframe = pl->nend - pl->nstart + 1;
  if (pl->nframe < 2) return set_err(MC_E_ARG, "need at least two frames (nStart %d, nEnd %d)", pl->nstart, pl->nend);
  int dist = pl->nframe / 2 - p.FrameDistOffset;
  if (dist <= 0) dist = 1;
  if (dist > pl->nframe / 2) dist = pl->nframe / 2;
  std::vector<mc::PairIJ> pairs;
  for (int i = 0; i < pl->nframe; i++)
    for (int j = i + dist; j < pl->nframe; j++) pairs.push_back({i, j});
  if (pl->cap_frames && (pl->nframe > pl->cap_frames || (int)pairs.size() > pl->cap_pairs))
    return set_err(MC_E_SIZE, "%d frames / %d pairs exceed the plan's capacity (%d / %d)", pl->nframe,
                   (int)pairs.size(), pl->cap_frames, pl->cap_pairs);
  const bool same = pairs == pl->pairs;
  pl->pairs = pairs;
  if (pl->d_pairs_main && !same && upload_pairs) {
    std::vector<int2> pr(pairs.size());
    for (size_t i = 0; i < pairs.size(); i++) pr[i] = make_int2(pairs[i].first, pairs[i].second);
    CK(cudaMemcpyAsync(pl->d_pairs_main, pr.data(), sizeof(int2) * pr.size(), cudaMemcpyHostToDevice, pl->st));
    CK(cudaStreamSynchronize(pl->st));
  }
  pl->loaded.assign(pl->nframe, 0);
  pl->frames_src = nullptr;
  pl->have_forward = pl->have_pairs = pl->have_solve = pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

static int create_plan(const mc_params* pin, int nx, int ny, int nz, int mode, int cap_frames, int cap_pairs,
                       int slots, mc_plan** out);

extern "C" {

int mc_plan_create(const mc_params* pin, int nx, int ny, int nz, int mode, mc_plan** out) {
  return create_plan(pin, nx, ny, nz, mode, 0, 0, 0, out);
}

int mc_plan_create_capacity(const mc_params* pin, int nx, int ny, int nz, int mode, int cap_frames, int cap_pairs,
                            mc_plan** out) {
  if (cap_frames < 0 || cap_pairs < 0) return set_err(MC_E_ARG, "negative capacity");
  return create_plan(pin, nx, ny, nz, mode, cap_frames, cap_pairs, 0, out);
}

int mc_plan_create_slots(const mc_params* pin, int nx, int ny, int nz, int mode, int cap_frames, int cap_pairs,
                         int slots, mc_plan** out) {
  if (cap_frames < 0 || cap_pairs < 0) return set_err(MC_E_ARG, "negative capacity");
  if (slots < 0 || (slots > 0 && slots < kMinSlots))
    return set_err(MC_E_ARG, "spectrum slots %d: 0 (automatic) or at least %d", slots, kMinSlots);
  return create_plan(pin, nx, ny, nz, mode, cap_frames, cap_pairs, slots, out);
}

int mc_schedule_set(const mc_schedule* s) {
  if (!s) return set_err(MC_E_ARG, "null schedule");
  if (s->n < 16 || s->pair_q < 0 || s->pairs_per_cta < 0 || s->pair_variant != 0 || s->fwd_streams < 0 ||
      s->fwd_streams > 8 || s->fwd_rows_pairing < 0 || s->fwd_rows_pairing > 2 || s->fwd_cols_pairing < 0 ||
      s->fwd_cols_pairing > 2)
    return set_err(MC_E_ARG, "bad schedule for n=%d", s->n);
  if (s->pair_q > 1 && (s->n % s->pair_q || !mc::pair_cols_reg_supported(s->n / s->pair_q, s->pair_q)))
    return set_err(MC_E_ARG, "pair stage takes no split %d = %d * %d", s->n, s->n / std::max(s->pair_q, 1),
                   s->pair_q);
  std::lock_guard<std::mutex> lk(g_sched_mu);
  g_sched[s->n] = *s;
  return MC_OK;
}

int mc_schedule_get(int n, mc_schedule* out) {
  if (!out) return set_err(MC_E_ARG, "null argument");
  if (!find_schedule(n, out)) return set_err(MC_E_ARG, "no schedule set for n=%d", n);
  return MC_OK;
}

void mc_schedule_clear(void) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  g_sched.clear();
}

int mc_schedule_candidates(int n, int* q_out, int max) {
  int c = 0;
  for (int q = 2; q <= n; q++) {
    if (n % q || !mc::pair_cols_reg_supported(n / q, q)) continue;
    if (q_out && c < max) q_out[c] = q;
    c++;
  }
  return c;
}

int mc_plan_reframe(mc_plan* pl, const mc_params* p, int nz) {
  if (!pl || !p) return set_err(MC_E_ARG, "null argument");
  if (nz <= 1) return set_err(MC_E_ARG, "Not a stack or wrong file. Abort");
  const mc_params& g = pl->p;
  if (p->crop_offsetx != g.crop_offsetx || p->crop_offsety != g.crop_offsety || p->crop_nsam != g.crop_nsam ||
      std::fabs(p->bin - pl->binf) > 1e-4f || p->CCPeakSearchDim != g.CCPeakSearchDim ||
      p->bfactor != g.bfactor || p->NoisePeakSize != g.NoisePeakSize || p->GPUNum != g.GPUNum)
    return set_err(MC_E_ARG, "reframe changes the plan geometry; create a new plan");
  CK(cudaSetDevice(pl->device));
  pl->p.iter = p->iter;
  pl->p.iterthres = p->iterthres;
  pl->p.refine = p->refine;
  return configure_frames(pl, *p, nz);
}

}  // extern "C"

static int create_plan(const mc_params* pin, int nx, int ny, int nz, int mode, int cap_frames, int cap_pairs,
                       int slots, mc_plan** out) {
  if (!pin || !out) return set_err(MC_E_ARG, "null argument");
  *out = nullptr;
  if (nx <= 0 || ny <= 0 || nz <= 0) return set_err(MC_E_ARG, "bad stack size %d x %d x %d", nx, ny, nz);
  if (word_length(mode) == 0) return set_err(MC_E_ARG, "unsupported MRC mode %d", mode);
  mc_plan* pl = new mc_plan();
  std::unique_ptr<mc_plan> guard(pl);
  pl->p = *pin;
  mc_params& p = pl->p;
  // bin clamp of getPara (dosefgpu_driftcorr.cpp:174-190)
  if (p.bin > 2.0001f) p.bin = 2.0f;
  else if (p.bin < 0.9999f) p.bin = 1.0f;
  pl->binf = p.bin;
  pl->nx = nx;
  pl->ny = ny;
  pl->nz = nz;
  pl->mode = mode;
  pl->wl = word_length(mode);
  pl->device = p.GPUNum;
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (p.GPUNum < 0 || p.GPUNum >= ndev)
    return set_err(MC_E_ARG, "GPU ID %d is out of range(%d). Abort.", p.GPUNum, ndev);
  CK(cudaSetDevice(p.GPUNum));
  // geometry (DFAlign.cu:500-530)
  pl->nu = verify_crop_size(nx, ny, p.crop_offsetx, p.crop_offsety, p.crop_nsam, p.bin);
  if (pl->nu <= 0) return set_err(MC_E_ARG, "Error: Wrong image Size.");
  pl->n = (int)((float)pl->nu / p.bin) / 2 * 2;
  if (pl->n < 16) return set_err(MC_E_SIZE, "binned size %d below 16", pl->n);
  pl->box = p.CCPeakSearchDim;
  if (pl->box < 16 || pl->box > 256 || pl->box > pl->n)
    return set_err(MC_E_SIZE, "-pbx %d outside [16, min(256, %d)]", pl->box, pl->n);
  if (pl->nu > 9216) return set_err(MC_E_SIZE, "crop side %d above 9216", pl->nu);
  pl->H = pl->n / 2 + 1;
  pl->ldn = (int)round_up(pl->n, 4);
  pl->ldu = (pl->nu == pl->n) ? pl->ldn : (int)round_up(pl->nu, 4);
  pl->ldt2 = (int)round_up(pl->H, 4);
  pl->fstride = (long long)pl->H * pl->ldn;
  const int ori = (pl->n - pl->box) / 2;
  pl->ystart = (ori + pl->n / 2) % pl->n;
  if (!make_plan(pl->nu, pl->plan_nu) || !make_plan(pl->n, pl->plan_n))
    return set_err(MC_E_SIZE, "no FFT plan for %d / %d", pl->nu, pl->n);
  choose_prune(pl->n, pl->box, pl->P, pl->Q);
  if (!make_plan(pl->Q, pl->plan_q)) return set_err(MC_E_SIZE, "no FFT plan for Q=%d", pl->Q);
  {
    const bool reg = mc::pair_cols_reg_supported(pl->P, pl->Q);
    const int team = pl->P <= 32 ? 32 : (pl->P <= 64 ? 64 : 128);
    const size_t need = std::max(mc::pair_cols_launch_smem(pl->n, pl->P, pl->Q, pl->box),
                                 reg ? mc::pair_cols_reg_smem(pl->n, team) : (size_t)0);
    if (need > 227 * 1024) return set_err(MC_E_SIZE, "pair stage does not fit shared memory for n=%d", pl->n);
    mc_schedule sc{};
    const bool have_sc = find_schedule(pl->n, &sc);
    pl->ppc = (have_sc && sc.pairs_per_cta > 0) ? std::min(sc.pairs_per_cta, 512) : kPairsPerCta;
    if (have_sc) {
      if (sc.fwd_streams > 0) pl->nfs = std::min(sc.fwd_streams, (int)mc_plan::kMaxForwardStreams);
      pl->fwd_rows_pairing = sc.fwd_rows_pairing;
      pl->fwd_cols_pairing = sc.fwd_cols_pairing;
    }
  }

  CK(cudaStreamCreateWithFlags(&pl->st, cudaStreamNonBlocking));
  for (auto& e : pl->ev) CK(cudaEventCreate(&e));

  // frame range and pair list; capacities default to this run's sizes
  CKR(configure_frames(pl, p, nz));
  pl->cap_frames = std::max(cap_frames, pl->nframe);
  pl->cap_pairs = std::max(cap_pairs, (int)pl->pairs.size());
  pl->maxp = std::max(pl->cap_pairs, pl->cap_frames);
  const int capf = pl->cap_frames;

  // device buffers
  pl->frame_bytes = (size_t)nx * ny * pl->wl;
  CKR(pl->alloc(&pl->d_frames, pl->frame_bytes * capf));
  if (pl->nu != pl->n) CKR(pl->alloc(&pl->d_T, sizeof(float2) * (size_t)pl->H * pl->ldu));
  CKR(pl->alloc(&pl->d_pairs, sizeof(int2) * pl->maxp));
  CKR(pl->alloc(&pl->d_G, sizeof(float2) * (size_t)std::min(pl->maxp, kPairBatch) * pl->H * pl->box));
  CKR(pl->alloc(&pl->d_boxes, sizeof(float) * (size_t)pl->maxp * pl->box * pl->box));
  CKR(pl->alloc(&pl->d_pshift, sizeof(float) * 2 * pl->maxp));
  CKR(pl->alloc(&pl->d_pcc, sizeof(float) * pl->maxp));
  CKR(pl->alloc(&pl->d_ppeak, sizeof(int) * 2 * pl->maxp));
  CKR(pl->alloc(&pl->d_sum, sizeof(float2) * pl->fstride));
  CKR(pl->alloc(&pl->d_T2, sizeof(float2) * (size_t)pl->n * pl->ldt2));
  {
    // image sums of two-level sizes accumulate into d_sumacc, then transform
    // (other sizes run the single fused kernel)
    int n1, n2;
    if (mc::two_level_split(pl->n, n1, n2))
      CKR(pl->alloc(&pl->d_sumacc, sizeof(float2) * pl->fstride));
  }
  CKR(pl->alloc(&pl->d_ey, sizeof(float2) * (size_t)capf * pl->n));
  CKR(pl->alloc(&pl->d_image, sizeof(float) * (size_t)pl->n * pl->n));
  CKR(pl->alloc(&pl->d_sumframes, sizeof(int) * capf));
  CKR(pl->alloc(&pl->d_apply, sizeof(int) * capf));
  CKR(pl->alloc(&pl->d_sumshift, sizeof(double2) * capf));
  CKR(pl->alloc(&pl->d_opart, sizeof(double) * ((size_t)pl->H * capf * 5 + pl->H)));
  CKR(pl->alloc(&pl->d_oout, sizeof(double) * ((size_t)capf * 5 + 1)));
  {
    // device-only pipeline: pair list, solve scratch and pinned result staging
    const int np = pl->cap_pairs, nf = capf, nc = nf - 1;
    std::vector<int2> pr(pl->pairs.size());
    for (size_t i = 0; i < pr.size(); i++) pr[i] = make_int2(pl->pairs[i].first, pl->pairs[i].second);
    CKR(pl->alloc(&pl->d_pairs_main, sizeof(int2) * np));
    CKR(upload(pl, pl->d_pairs_main, pr));
    CKR(pl->alloc(&pl->d_M, sizeof(double) * (size_t)nc * nc));
    CKR(pl->alloc(&pl->d_rhs, sizeof(double) * 2 * (size_t)nc));
    CKR(pl->alloc(&pl->d_work, sizeof(double) * (2 * (size_t)nc + 2 * (size_t)nf)));
    CKR(pl->alloc(&pl->d_ki1, sizeof(double) * np));
    CKR(pl->alloc(&pl->d_ki2, sizeof(double) * np));
    CKR(pl->alloc(&pl->d_dshift, sizeof(double) * 2 * (size_t)nc));
    CKR(pl->alloc(&pl->d_dfshift, sizeof(double) * 2 * (size_t)nf));
    CKR(pl->alloc(&pl->d_mask, sizeof(int) * np));
    CKR(pl->alloc(&pl->d_order, sizeof(int) * np));
    CKR(pl->alloc(&pl->d_uf, sizeof(int) * nf));
    CKR(pl->alloc(&pl->d_kept, sizeof(int) * np));
    CKR(pl->alloc(&pl->d_nkept, sizeof(int)));
    CKR(pl->alloc(&pl->d_status, sizeof(int)));
    size_t o = 0;
    auto place = [&](size_t& off, size_t bytes) {
      off = o;
      o += (bytes + 15) / 16 * 16;
    };
    place(pl->st_dc, sizeof(float2) * nf);
    place(pl->st_pshift, sizeof(float) * 2 * np);
    place(pl->st_pcc, sizeof(float) * np);
    place(pl->st_ppeak, sizeof(int) * 2 * np);
    place(pl->st_ki1, sizeof(double) * np);
    place(pl->st_kept, sizeof(int) * np);
    place(pl->st_nkept, sizeof(int));
    place(pl->st_ki2, sizeof(double) * np);
    place(pl->st_work, sizeof(double) * 2 * (size_t)nc);
    place(pl->st_status, sizeof(int));
    place(pl->st_slot, sizeof(void*));
    pl->st_bytes = o;
    if (injected_alloc_failure())
      return set_err(MC_E_NOMEM, "cudaMallocHost(%zu bytes) failed: injected failure (mc_debug_fail_alloc)", o);
    CK(cudaMallocHost(&pl->h_stage, o));
    CKR(pl->alloc(&pl->d_src_slot, sizeof(void*)));
  }

  // tables
  CKR(pl->alloc(&pl->d_tw_nu, sizeof(float2) * pl->nu));
  CKR(upload(pl, pl->d_tw_nu, twiddles(pl->nu, -1)));
  if (pl->nu == pl->n) {
    pl->d_tw_n = pl->d_tw_nu;
  } else {
    CKR(pl->alloc(&pl->d_tw_n, sizeof(float2) * pl->n));
    CKR(upload(pl, pl->d_tw_n, twiddles(pl->n, -1)));
  }
  CKR(pl->alloc(&pl->d_twQ, sizeof(float2) * pl->Q));
  CKR(upload(pl, pl->d_twQ, twiddles(pl->Q, -1)));
  if (!mc::pair_cols_reg_supported(pl->P, pl->Q) && mc::pair_cols_tabn(pl->n, pl->P, pl->box)) {
    // generic column kernel with a length-n outer table: exp(+2 pi i e / n)
    std::vector<float2> tn(pl->n);
    for (int e = 0; e < pl->n; e++) {
      const double ang = 2.0 * kPi * (double)e / pl->n;
      tn[e] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    CKR(pl->alloc(&pl->d_twN, sizeof(float2) * tn.size()));
    CKR(upload(pl, pl->d_twN, tn));
  }
  {
    std::vector<float2> two((size_t)pl->P * pl->box);
    for (int k = 0; k < pl->P; k++)
      for (int m = 0; m < pl->box; m++) {
        const long long y = (pl->ystart + m) % pl->n;
        const long long e = ((long long)k * y) % pl->n;
        const double ang = 2.0 * kPi * (double)e / pl->n;
        two[(size_t)k * pl->box + m] = make_float2((float)std::cos(ang), (float)std::sin(ang));
      }
    CKR(pl->alloc(&pl->d_twO, sizeof(float2) * two.size()));
    CKR(upload(pl, pl->d_twO, two));
    std::vector<float2> cs((size_t)pl->H * pl->box);
    for (int k = 0; k < pl->H; k++) {
      const double h = (k == 0 || k == pl->n / 2) ? 1.0 : 2.0;
      for (int m = 0; m < pl->box; m++) {
        const long long x = (pl->ystart + m) % pl->n;
        const long long e = ((long long)k * x) % pl->n;
        const double ang = 2.0 * kPi * (double)e / pl->n;
        cs[(size_t)k * pl->box + m] = make_float2((float)(h * std::cos(ang)), (float)(h * std::sin(ang)));
      }
    }
    CKR(pl->alloc(&pl->d_cs, sizeof(float2) * cs.size()));
    CKR(upload(pl, pl->d_cs, cs));
    // cosmask2d weights (func.cpp:348-370)
    std::vector<double> w(16 * 9);
    for (int j = 0; j < 16; j++) {
      const int ky = j < 8 ? j : j - 16;
      for (int i = 0; i < 9; i++) {
        const int r = (int)std::sqrt((float)(i * i + ky * ky));
        w[j * 9 + i] = r < 8 ? std::cos(r * kPi / 8.0) / 2 + 0.5 : 0.0;
      }
    }
    CKR(pl->alloc(&pl->d_w16, sizeof(double) * w.size()));
    CKR(upload(pl, pl->d_w16, w));
  }
  {
    // the spectrum store, last: every frame position's spectrum, or `slots`
    // of them when asked or when the free device memory holds fewer
    const size_t spec = sizeof(float2) * (size_t)pl->fstride;
    int ns = capf;
    if (slots > 0) {
      ns = std::min(slots, capf);
    } else {
      size_t fr = 0, tot = 0;
      CK(cudaMemGetInfo(&fr, &tot));
      const size_t budget = g_device_budget.load();
      if (budget) fr = std::min(fr, budget);
      const size_t room = fr > kKeepFree ? fr - kKeepFree : 0;
      if ((size_t)capf * spec > room) {
        ns = (int)std::min<size_t>(room / spec, (size_t)capf);
        if (ns < kMinSlots)
          return set_err(MC_E_NOMEM,
                         "%d spectra of %zu bytes do not fit the free device memory (%zu bytes), nor do %d of them",
                         capf, spec, fr, kMinSlots);
      }
    }
    CKR(pl->alloc(&pl->d_specA, spec * ns));
    pl->d_specB = pl->d_specA;
    if (ns < capf) {
      pl->slots = ns;
      pl->slot_frame.assign(ns, -1);
      pl->slot_use.assign(ns, 0);
      pl->frame_slot.assign(capf, -1);
    }
  }
  CK(cudaStreamSynchronize(pl->st));
  pl->loaded.assign(pl->nframe, 0);
  *out = guard.release();
  return MC_OK;
}

// Forget the captured movie graphs (their kernels hold the reference and
// frame-source pointers of the configuration they were captured with).
static void drop_graphs(mc_plan* pl) {
  if (pl->st) cudaStreamSynchronize(pl->st);
  for (auto& g : pl->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  pl->graphs.clear();
}

// The references gathered through the stretch maps (first use allocates).
static int stretch_refs(mc_plan* pl) {
  if (!pl->stretch) return MC_OK;
  const size_t bytes = sizeof(float) * (size_t)pl->nx * pl->ny;
  auto one = [&](const float* src, float** dst) -> int {
    if (!src) return MC_OK;
    if (!*dst) CKR(pl->alloc(dst, bytes));
    CK(mc::launch_stretch_full(src, *dst, pl->d_rmap, pl->d_cmap, pl->nx, pl->ny, pl->st));
    return MC_OK;
  };
  CKR(one(pl->d_dark, &pl->d_dark_s));
  CKR(one(pl->d_dark2, &pl->d_dark2_s));
  CKR(one(pl->d_norm, &pl->d_norm_s));
  CKR(one(pl->d_norm2, &pl->d_norm2_s));
  CK(cudaStreamSynchronize(pl->st));
  return MC_OK;
}

extern "C" {

int mc_plan_info(const mc_plan* pl, mc_info* i) {
  if (!pl || !i) return set_err(MC_E_ARG, "null argument");
  i->nx = pl->nx;
  i->ny = pl->ny;
  i->nz = pl->nz;
  i->mode = pl->mode;
  i->nsam_unbin = pl->nu;
  i->nsam = pl->n;
  i->nstart = pl->nstart;
  i->nend = pl->nend;
  i->nframe = pl->nframe;
  i->npairs = (int)pl->pairs.size();
  i->two_sets = pl->two_sets ? 1 : 0;
  i->prune_p = pl->P;
  i->prune_q = pl->Q;
  i->device_bytes = pl->dev_bytes;
  i->spectrum_slots = pl->slots;
  i->forward_recomputes = pl->recomputes;
  return MC_OK;
}

int mc_plan_set_refs(mc_plan* pl, const float* dark, const float* dark2, const float* norm, const float* norm2) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  CK(cudaSetDevice(pl->device));
  const size_t bytes = sizeof(float) * (size_t)pl->nx * pl->ny;
  auto put = [&](float** d, const float* h) -> int {
    if (!h) {
      *d = nullptr;
      return MC_OK;
    }
    float* q = nullptr;
    CKR(pl->alloc(&q, bytes));
    CK(cudaMemcpyAsync(q, h, bytes, cudaMemcpyHostToDevice, pl->st));
    *d = q;
    return MC_OK;
  };
  if ((dark2 && !dark) || (norm2 && !norm)) return set_err(MC_E_ARG, "second reference without the first");
  CKR(put(&pl->d_dark, dark));
  CKR(put(&pl->d_dark2, dark2));
  CKR(put(&pl->d_norm, norm));
  CKR(put(&pl->d_norm2, norm2));
  const bool two = dark || norm;
  if (two && !pl->two_sets) {
    // as many spectra as set A holds (a reframe may grow nframe up to cap_frames)
    CKR(pl->alloc(&pl->d_specB, sizeof(float2) * pl->fstride * (pl->slots ? pl->slots : pl->cap_frames)));
    pl->two_sets = true;
  }
  CK(cudaStreamSynchronize(pl->st));
  CKR(stretch_refs(pl));
  drop_graphs(pl);  // captured movies hold the previous reference pointers
  pl->have_forward = pl->have_pairs = pl->have_solve = pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

// -scx/-scy (DFAlign.cu:503-504, 751-765).
int mc_plan_set_stretch(mc_plan* pl, float xscale, float yscale) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!(xscale >= 1.0f)) return set_err(MC_E_ARG, "Stretching factor along X-axis needs to be >=1.0.");
  if (!(yscale >= 1.0f)) return set_err(MC_E_ARG, "Stretching factor along Y-axis needs to be >=1.0.");
  CK(cudaSetDevice(pl->device));
  const float xs = (float)(1.0 / xscale), ys = (float)(1.0 / yscale);
  const bool on = xs < 1.0f || ys < 1.0f;
  if (on) {
    // addr_orig = int(ky*yscale+0.5)*nx + int(kx*xscale+0.5): float product, double sum
    auto map = [](int len, float s) {
      std::vector<int> m(len);
      for (int k = 0; k < len; k++) m[k] = std::min(len - 1, std::max(0, (int)((double)((float)k * s) + 0.5)));
      return m;
    };
    const std::vector<int> rm = map(pl->ny, ys), cm = map(pl->nx, xs);
    if (!pl->d_rmap) {
      CKR(pl->alloc(&pl->d_rmap, sizeof(int) * (size_t)pl->ny));
      CKR(pl->alloc(&pl->d_cmap, sizeof(int) * (size_t)pl->nx));
      CKR(pl->alloc(&pl->d_sframe, pl->frame_bytes));
    }
    CK(cudaMemcpyAsync(pl->d_rmap, rm.data(), sizeof(int) * rm.size(), cudaMemcpyHostToDevice, pl->st));
    CK(cudaMemcpyAsync(pl->d_cmap, cm.data(), sizeof(int) * cm.size(), cudaMemcpyHostToDevice, pl->st));
  }
  pl->stretch = on;
  CKR(stretch_refs(pl));
  drop_graphs(pl);
  pl->have_forward = pl->have_pairs = pl->have_solve = pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

static int load_frames(mc_plan* pl, const void* src, int first, int count, cudaMemcpyKind kind) {
  if (!pl || !src) return set_err(MC_E_ARG, "null argument");
  if (first < 0 || count < 0 || first + count > pl->nframe)
    return set_err(MC_E_ARG, "frames [%d, %d) outside [0, %d)", first, first + count, pl->nframe);
  CK(cudaSetDevice(pl->device));
  CK(cudaMemcpyAsync((char*)pl->d_frames + (size_t)first * pl->frame_bytes, src, (size_t)count * pl->frame_bytes,
                     kind, pl->st));
  // the caller may reuse a host buffer as soon as this returns
  if (kind == cudaMemcpyHostToDevice) CK(cudaStreamSynchronize(pl->st));
  if (pl->frames_src) {
    // back to the plan's own frame buffer: nothing of it is loaded yet
    pl->frames_src = nullptr;
    pl->loaded.assign(pl->nframe, 0);
  }
  for (int i = first; i < first + count; i++) pl->loaded[i] = 1;
  pl->have_forward = pl->have_pairs = pl->have_solve = pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

int mc_plan_load_frames(mc_plan* pl, const void* frames, int first, int count) {
  return load_frames(pl, frames, first, count, cudaMemcpyHostToDevice);
}

int mc_plan_load_frames_device(mc_plan* pl, const void* d_frames, int first, int count) {
  return load_frames(pl, d_frames, first, count, cudaMemcpyDeviceToDevice);
}

int mc_plan_bind_frames_device(mc_plan* pl, const void* d_frames) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (d_frames) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, d_frames) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
        at.device != pl->device) {
      cudaGetLastError();
      return set_err(MC_E_ARG, "bound frames are not device memory of GPU %d", pl->device);
    }
  }
  pl->frames_src = d_frames;
  pl->loaded.assign(pl->nframe, d_frames ? 1 : 0);
  pl->have_forward = pl->have_pairs = pl->have_solve = pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

}  // extern "C"

static int run_device(mc_plan* pl, float* image_host, const std::vector<cudaEvent_t>* waits, int chunk);
static bool device_path(const mc_plan* pl);

// Forward transforms of every position.  With `waits`, the plan stream waits
// for (*waits)[f / chunk] before the first frame of each chunk (pipelined
// upload); the per-frame means are read back and logged at the end.
static int enqueue_forward(mc_plan* pl, const std::vector<cudaEvent_t>* waits, int chunk,
                           const std::vector<std::pair<int, int>>* only) {
  // `only`: (frame, spectrum slot) pairs to transform (the spectra-slot mode);
  // default every frame into its own slot
  const bool binned = pl->nu != pl->n;
  // frames write only their own spectrum slots unless a shared scratch is in
  // play (binning's row buffer, the stretched frame); per-launch timing
  // events need the one stream
  const int njob = only ? (int)only->size() : pl->nframe;
  const bool multi = !binned && !pl->stretch && njob > 1 && !(pl->profiling && !pl->capturing);
  const int NS = pl->nfs;
  if (multi) {
    for (int i = 0; i < NS; i++) {
      if (!pl->fst[i]) CK(cudaStreamCreateWithFlags(&pl->fst[i], cudaStreamNonBlocking));
      if (!pl->fev[i]) CK(cudaEventCreateWithFlags(&pl->fev[i], cudaEventDisableTiming));
    }
    cudaEvent_t& fork = pl->fev[mc_plan::kMaxForwardStreams];
    if (!fork) CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CK(cudaEventRecord(fork, pl->st));
    for (int i = 0; i < NS; i++) CK(cudaStreamWaitEvent(pl->fst[i], fork, 0));
  }
  for (int job = 0; job < njob; job++) {
    const int f = only ? (*only)[job].first : job;
    const int slot = only ? (*only)[job].second : job;
    cudaStream_t fs = multi ? pl->fst[job % NS] : pl->st;
    if (waits && (multi || f % chunk == 0)) CK(cudaStreamWaitEvent(fs, (*waits)[f / chunk], 0));
    mc::FwdRowsArgs a{};
    a.frame = (const char*)(pl->frames_src ? pl->frames_src : pl->d_frames) + (size_t)f * pl->frame_bytes;
    a.frames_slot = pl->d_src_slot;
    a.frame_offset = (long long)f * (long long)pl->frame_bytes;
    if (pl->stretch) {
      // the crop of this frame through the stretch maps, then transformed from there
      LAUNCH(pl, MC_K_FWD_ROWS, 2.0 * pl->nu * pl->nu * pl->wl,
             mc::launch_stretch_crop(pl->d_src_slot, a.frame_offset, a.frame, pl->wl, pl->d_sframe, pl->d_rmap,
                                     pl->d_cmap, pl->nx, pl->p.crop_offsetx, pl->p.crop_offsety, pl->nu, fs));
      a.frame = pl->d_sframe;
      a.frames_slot = nullptr;
      a.frame_offset = 0;
    }
    a.mode = pl->mode;
    a.nx = pl->nx;
    a.ny = pl->ny;
    a.offx = pl->p.crop_offsetx;
    a.offy = pl->p.crop_offsety;
    a.nu = pl->nu;
    a.hk = pl->H;
    const bool stretched = pl->stretch;
    a.dark = stretched ? pl->d_dark_s : pl->d_dark;
    a.dark2 = stretched ? pl->d_dark2_s : pl->d_dark2;
    a.norm = stretched ? pl->d_norm_s : pl->d_norm;
    a.norm2 = stretched ? pl->d_norm2_s : pl->d_norm2;
    a.two_outputs = pl->two_sets ? 1 : 0;
    float2* TA = binned ? pl->d_T : specA_at(pl, slot);
    a.outA = TA;
    a.ldt = binned ? pl->ldu : pl->ldn;
    a.plan = pl->plan_nu;
    a.tw = pl->d_tw_nu;
    const int nrefs = (pl->d_dark ? 1 : 0) + (pl->d_dark2 ? 1 : 0) + (pl->d_norm ? 1 : 0) + (pl->d_norm2 ? 1 : 0);
    const double crop_bytes = (double)pl->nu * pl->nu * (pl->wl + 4.0 * nrefs);
    const double t_bytes = (double)pl->H * pl->nu * sizeof(float2);
    const double s_bytes = (double)pl->H * pl->n * sizeof(float2);
    float2* TB = nullptr;
    if (pl->two_sets) TB = binned ? nullptr : specB_at(pl, slot);
    if (pl->two_sets && binned) {
      // binned two-set case: set A, then set B, each through the scratch d_T
      // with its references folded into the one-output row transform
      for (int set = 0; set < 2; set++) {
        mc::FwdRowsArgs b = a;
        b.two_outputs = 0;
        b.dark = set == 0 ? a.dark : a.dark2;
        b.norm = set == 0 ? a.norm : a.norm2;
        b.dark2 = nullptr;
        b.norm2 = nullptr;
        b.outA = pl->d_T;
        b.paired = pl->fwd_rows_pairing;
        LAUNCH(pl, MC_K_FWD_ROWS, crop_bytes + t_bytes, mc::launch_fwd_rows(b, fs));
        mc::RowsFftArgs c{};
        c.in = pl->d_T;
        c.ld_in = pl->ldu;
        c.out = set == 0 ? specA_at(pl, slot) : specB_at(pl, slot);
        c.ld_out = pl->ldn;
        c.nrows = pl->H;
        c.n_out = pl->n;
        c.keep_lo = pl->n / 2;
        c.scale = 1.f;
        c.plan = pl->plan_nu;
        c.tw = pl->d_tw_nu;
        c.paired = pl->fwd_cols_pairing;
        LAUNCH(pl, MC_K_FWD_COLS, t_bytes + s_bytes, mc::launch_rows_fft(c, false, 1, fs));
      }
      continue;
    }
    a.outB = TB;
    a.paired = pl->fwd_rows_pairing;
    LAUNCH(pl, MC_K_FWD_ROWS, crop_bytes + t_bytes * (pl->two_sets ? 2 : 1), mc::launch_fwd_rows(a, fs));
    for (int set = 0; set < (pl->two_sets ? 2 : 1); set++) {
      mc::RowsFftArgs c{};
      c.in = set == 0 ? TA : TB;
      c.ld_in = a.ldt;
      c.out = set == 0 ? specA_at(pl, slot) : specB_at(pl, slot);
      c.ld_out = pl->ldn;
      c.nrows = pl->H;
      c.n_out = pl->n;
      c.keep_lo = binned ? pl->n / 2 : pl->n;
      c.scale = 1.f;
      c.plan = pl->plan_nu;
      c.tw = pl->d_tw_nu;
      c.paired = pl->fwd_cols_pairing;
      LAUNCH(pl, MC_K_FWD_COLS, t_bytes + s_bytes, mc::launch_rows_fft(c, false, 1, fs));
    }
  }
  if (multi)
    for (int i = 0; i < NS; i++) {
      CK(cudaEventRecord(pl->fev[i], pl->fst[i]));
      CK(cudaStreamWaitEvent(pl->st, pl->fev[i], 0));
    }
  return MC_OK;
}

// pair lines (DFAlign.cu:903-904)
static void log_pairs(mc_plan* pl) {
  pl->log("\nCalculate relative drift between frames\n");
  for (size_t j = 0; j < pl->pairs.size(); j++)
    pl->log("......%03d Frame #%03d VS #%03d xy-shift: %8.4f %8.4f      CC:%f\n", (int)j,
            pl->pairs[j].first + pl->nstart, pl->pairs[j].second + pl->nstart, pl->pshift[2 * j],
            pl->pshift[2 * j + 1], pl->pcc[j]);
}

// ki lines of both rounds (DFAlign.cu:917-948)
static void log_solve(mc_plan* pl) {
  const int np = (int)pl->pairs.size();
  pl->log("\n......ki: First round \n");
  double acc = 0;
  for (int j = 0; j < np; j++) {
    pl->log("......ki #%03d of Frame #%03d VS #%03d: %8.4lf \n", j + pl->nstart, pl->pairs[j].first + pl->nstart,
            pl->pairs[j].second + pl->nstart, pl->ki1[j]);
    acc += pl->ki1[j];
  }
  pl->log("................................Average ki: %8.4lf \n\n", acc / np);
  pl->log("......ki: Second round \n");
  acc = 0;
  for (size_t j = 0; j < pl->good.size(); j++) {
    const auto& pr = pl->pairs[pl->good[j]];
    pl->log("......ki #%03d of Frame #%03d VS #%03d: %8.4f \n", (int)j + pl->nstart, pr.first + pl->nstart,
            pr.second + pl->nstart, pl->ki2[j]);
    acc += pl->ki2[j];
  }
  pl->log("................................Average ki: %8.4lf \n\n", acc / (double)pl->good.size());
}

// per-frame mean: Re F(0,0) / n / n (DFAlign.cu:818), from the DC terms
static void log_frame_means(mc_plan* pl, const float2* dc) {
  pl->frame_mean.resize(pl->nframe);
  pl->log("\nRead stack:\n");
  for (int f = 0; f < pl->nframe; f++) {
    pl->frame_mean[f] = dc[f].x / pl->n / pl->n;
    pl->log("......Read and sum frame #%03d   mean:%f\n", f + pl->nstart, pl->frame_mean[f]);
  }
}

// Base of the run's frames (the plan's buffer or bound caller frames) into
// the device word the forward kernels read, ordered on the plan stream
// before them; outside any capture, so a captured movie serves every frame
// buffer.  The pinned source word is rewritten only after the previous
// movie synchronised.
static int upload_frame_base(mc_plan* pl) {
  const void** h = reinterpret_cast<const void**>(pl->h_stage + pl->st_slot);
  *h = pl->frames_src ? pl->frames_src : pl->d_frames;
  CK(cudaMemcpyAsync(pl->d_src_slot, h, sizeof(void*), cudaMemcpyHostToDevice, pl->st));
  return MC_OK;
}

static int forward_all(mc_plan* pl, const std::vector<cudaEvent_t>* waits, int chunk) {
  CKR(upload_frame_base(pl));
  CK(cudaEventRecord(pl->ev[0], pl->st));
  std::vector<float2> dc(pl->nframe);
  if (pl->slots) {
    // slot mode: every frame once, `slots` at a time, for its DC term; the
    // last chunk stays held for the stage that follows
    clear_slots(pl);
    if (waits)
      for (size_t c = 0; c * chunk < (size_t)pl->nframe; c++) CK(cudaStreamWaitEvent(pl->st, (*waits)[c], 0));
    float2* hdc = reinterpret_cast<float2*>(pl->h_stage + pl->st_dc);
    for (int f0 = 0; f0 < pl->nframe; f0 += pl->slots) {
      std::vector<int> fr, where;
      for (int f = f0; f < std::min(pl->nframe, f0 + pl->slots); f++) fr.push_back(f);
      CKR(hold_spectra(pl, fr, where, true));
      for (size_t i = 0; i < fr.size(); i++)
        CK(cudaMemcpyAsync(hdc + fr[i], specA_at(pl, where[i]), sizeof(float2), cudaMemcpyDeviceToHost, pl->st));
    }
    CK(cudaEventRecord(pl->ev[1], pl->st));
    CK(cudaStreamSynchronize(pl->st));
    std::copy(hdc, hdc + pl->nframe, dc.begin());
  } else {
    CKR(enqueue_forward(pl, waits, chunk));
    CK(cudaEventRecord(pl->ev[1], pl->st));
    CK(cudaMemcpy2DAsync(dc.data(), sizeof(float2), pl->d_specA, sizeof(float2) * pl->fstride, sizeof(float2),
                         pl->nframe, cudaMemcpyDeviceToHost, pl->st));
    CK(cudaStreamSynchronize(pl->st));
  }
  CKR(pl->collect());
  CK(cudaEventElapsedTime(&pl->tm.forward_ms, pl->ev[0], pl->ev[1]));
  log_frame_means(pl, dc.data());
  pl->have_forward = true;
  pl->have_pairs = pl->have_solve = pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

extern "C" {

int mc_plan_forward(mc_plan* pl) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  for (int f = 0; f < pl->nframe; f++)
    if (!pl->loaded[f]) return set_err(MC_E_STATE, "frame position %d not loaded", f);
  CK(cudaSetDevice(pl->device));
  return forward_all(pl, nullptr, 1);
}

int mc_plan_run_host(mc_plan* pl, const void* frames, float* image_host) {
  if (!pl || !frames) return set_err(MC_E_ARG, "null argument");
  CK(cudaSetDevice(pl->device));
  if (!pl->st_copy) CK(cudaStreamCreateWithFlags(&pl->st_copy, cudaStreamNonBlocking));
  // chunks of frames: copy chunk c on the copy stream while the plan stream
  // transforms the frames of chunks < c
  const int chunk = 4;
  const int nchunk = (pl->nframe + chunk - 1) / chunk;
  while ((int)pl->chunk_ev.size() < nchunk) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    pl->chunk_ev.push_back(e);
  }
  // the copies start after everything already queued on the plan stream
  // (earlier readers of d_frames, a caller's start event)
  if (!pl->start_ev) CK(cudaEventCreateWithFlags(&pl->start_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(pl->start_ev, pl->st));
  CK(cudaStreamWaitEvent(pl->st_copy, pl->start_ev, 0));
  pl->frames_src = nullptr;
  for (int c = 0; c < nchunk; c++) {
    const int f0 = c * chunk, cnt = std::min(chunk, pl->nframe - f0);
    CK(cudaMemcpyAsync((char*)pl->d_frames + (size_t)f0 * pl->frame_bytes,
                       (const char*)frames + (size_t)f0 * pl->frame_bytes, (size_t)cnt * pl->frame_bytes,
                       cudaMemcpyHostToDevice, pl->st_copy));
    CK(cudaEventRecord(pl->chunk_ev[c], pl->st_copy));
  }
  for (int f = 0; f < pl->nframe; f++) pl->loaded[f] = 1;
  pl->log("Input Stack: Nx(%d) Ny(%d) Nz(%d) Mode(%d)\n\n", pl->nx, pl->ny, pl->nz, pl->mode);
  pl->log("Crop Image: Offset(%d %d) RawDim(%d) BinnedDim(%d)\n", pl->p.crop_offsetx, pl->p.crop_offsety, pl->nu,
          pl->n);
  if (device_path(pl)) return run_device(pl, image_host, &pl->chunk_ev, chunk);
  CKR(forward_all(pl, &pl->chunk_ev, chunk));
  CKR(mc_plan_pairs(pl));
  CKR(mc_plan_solve(pl));
  CKR(mc_plan_iterate(pl));
  pl->tm.refine_ms = 0.f;
  if (pl->p.refine) CKR(mc_plan_refine(pl, 4));
  CKR(mc_plan_sum(pl, image_host));
  pl->tm.total_ms = pl->tm.forward_ms + pl->tm.pairs_ms + pl->tm.iterate_ms + pl->tm.refine_ms + pl->tm.sum_ms;
  return MC_OK;
}

int mc_plan_pairs(mc_plan* pl) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_forward) return set_err(MC_E_STATE, "pairs before forward");
  CK(cudaSetDevice(pl->device));
  CK(cudaEventRecord(pl->ev[2], pl->st));
  CKR(run_pair_list(pl, pl->d_specA, pl->fstride, pl->d_specB, pl->fstride, pl->pairs, pl->pshift, pl->pcc,
                    pl->ppeak));
  CK(cudaEventRecord(pl->ev[3], pl->st));
  CK(cudaEventSynchronize(pl->ev[3]));
  CK(cudaEventElapsedTime(&pl->tm.pairs_ms, pl->ev[2], pl->ev[3]));
  log_pairs(pl);
  pl->have_pairs = true;
  pl->have_solve = pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

int mc_plan_solve(mc_plan* pl) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_pairs) return set_err(MC_E_STATE, "solve before pairs");
  const int np = (int)pl->pairs.size();
  const int ncol = pl->nframe - 1;
  std::vector<cplx> b(np);
  for (int j = 0; j < np; j++) b[j] = cplx(pl->pshift[2 * j], pl->pshift[2 * j + 1]);
  std::vector<int> all(np);
  for (int j = 0; j < np; j++) all[j] = j;
  std::vector<cplx> s;
  if (!mc::lsq_intervals(pl->pairs, all, ncol, b, s)) return set_err(MC_E_NUMERIC, "singular pair system");
  pl->ki1 = mc::lsq_residuals(pl->pairs, all, b, s);
  pl->good = mc::od_threshold(pl->pairs, pl->ki1, pl->nframe, (double)pl->p.kiThresh);
  if (!mc::lsq_intervals(pl->pairs, pl->good, ncol, b, s)) return set_err(MC_E_NUMERIC, "singular pair system");
  pl->ki2 = mc::lsq_residuals(pl->pairs, pl->good, b, s);
  log_solve(pl);
  pl->shift = s;
  pl->have_solve = true;
  pl->have_iter = pl->have_sum = false;
  return MC_OK;
}

int mc_plan_iterate(mc_plan* pl) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_solve) return set_err(MC_E_STATE, "iterate before solve");
  CK(cudaSetDevice(pl->device));
  const int nf = pl->nframe;
  std::vector<cplx>& shift = pl->shift;
  pl->log("Begin Iterative Alignment... \n");
  std::vector<cplx> newshift(nf);
  cplx all(0, 0);
  newshift[0] = 0;
  for (int j = 0; j < nf - 1; j++) {
    newshift[j + 1] = all + shift[j];
    all += shift[j];
  }
  std::vector<cplx> oldshift = newshift;
  double rmsd = 0;
  bool converged = false;
  int j;
  CK(cudaEventRecord(pl->ev[4], pl->st));
  std::vector<mc::PairIJ> fl(nf);
  for (int k = 0; k < nf; k++) fl[k] = {0, k};
  std::vector<int> frames(nf), apply(nf, 1);
  for (int k = 0; k < nf; k++) frames[k] = k;
  const float ith = pl->p.iterthres;
  for (j = 0; j < pl->p.iter && !converged; j++) {
    pl->log("Iteration [%d/%d]\n", j, pl->p.iter);
    std::vector<cplx> sh(nf);
    for (int k = 0; k < nf; k++) sh[k] = -oldshift[k];
    CKR(run_shift_sum(pl, frames, sh, apply, 0));
    for (int k = 0; k < nf; k++)
      pl->log("......Add Frame #%03d with xy shift: %8.4lf %8.4lf\n", k + pl->nstart, -oldshift[k].real(),
              -oldshift[k].imag());
    pl->log("Sum complete... \n");
    std::vector<float> fs, fc;
    std::vector<int> fp;
    CKR(run_pair_list(pl, pl->d_sum, 0, pl->d_specA, pl->fstride, fl, fs, fc, fp));
    double avgcc = 0;
    for (int k = 0; k < nf; k++) {
      newshift[k] = cplx(fs[2 * k], fs[2 * k + 1]);
      avgcc += fc[k];
      const cplx d = oldshift[k] - newshift[k];
      pl->log("......%03d Frame #%03d VS <sum> xy-shift: %8.4f %8.4f (%8.4f %8.4f) CC:%f\n", k, k + pl->nstart,
              fs[2 * k], fs[2 * k + 1], d.real(), d.imag(), fc[k]);
    }
    const cplx ref = newshift[0];
    for (int k = 0; k < nf; k++) {
      const cplx d = oldshift[k] - newshift[k];
      oldshift[k] = newshift[k] - ref;
      rmsd += d.real() * d.real() + d.imag() * d.imag();
    }
    pl->log("Average CC : %8.4f\n", avgcc / nf);
    rmsd /= nf;
    if (rmsd < (double)(ith * ith)) {
      converged = true;
      pl->log("Converged at iteration [%d/%d]\n", j, pl->p.iter);
    }
    pl->log("RMSD to <sum> : %8.4f  (%8.4f for convergence)\n", std::sqrt(rmsd), ith);
  }
  CK(cudaEventRecord(pl->ev[5], pl->st));
  CK(cudaEventSynchronize(pl->ev[5]));
  CK(cudaEventElapsedTime(&pl->tm.iterate_ms, pl->ev[4], pl->ev[5]));
  pl->log("Final RMSD to <sum> : %8.4f at iteration [%d/%d]\n\nShifts (delta) after iterative aligment\n",
          std::sqrt(rmsd), j - 1, pl->p.iter);
  pl->log("...Frame #%03d xy-shift %8.4f %8.4f (%8.4f %8.4f)\n", 0, 0.0, 0.0, 0.0, 0.0);
  all = 0;
  for (int k = 0; k < nf - 1; k++) {
    all += shift[k];
    const cplx td = all - oldshift[k + 1];
    pl->log("...Frame #%03d xy-shift %8.4f %8.4f (%8.4f %8.4f)\n", k + 1, oldshift[k + 1].real(),
            oldshift[k + 1].imag(), td.real(), td.imag());
    shift[k] = oldshift[k + 1] - oldshift[k];
  }
  pl->log("Final shift:\n");
  pl->frame_shift.assign(nf, cplx(0, 0));
  cplx total(0, 0);
  pl->log("......Shift of Frame #%03d : %8.4f %8.4f\n", pl->nstart, total.real(), total.imag());
  for (int k = 0; k < nf - 1; k++) {
    total = total + shift[k];
    pl->frame_shift[k + 1] = total;
    pl->log("......Shift of Frame #%03d : %8.4f %8.4f\n", k + pl->nstart + 1, total.real(), total.imag());
  }
  pl->have_iter = true;
  return MC_OK;
}

}  // extern "C"

// Frame range of the sum and the steps entering the middle-frame offset
// (DFAlign.cu:1115-1139); the reference reads past the shift vector when
// RefFrame - nStart > nframe - 1, here the offset stops at the last step.
static void sum_range(const mc_plan* pl, int* nss_out, int* nes_out, int* mid_steps) {
  const int nf = pl->nframe;
  const mc_params& p = pl->p;
  int nss = p.nStartSum - pl->nstart;
  int nes = p.nEndSum - pl->nstart;
  if (nss <= 0) nss = 0;
  if (nes <= nss || nes >= nf) nes = nf - 1;
  int lim = 0;
  if (p.bAlignToMid) {
    int ref = pl->nz / 2 + 1;
    if (ref < pl->nstart) ref = pl->nstart;
    lim = std::max(0, std::min(ref - pl->nstart, nf - 1));
  }
  *nss_out = nss;
  *nes_out = nes;
  *mid_steps = lim;
}

// Sum shifts s_k = -total_k + mid of the summed frames with the reference's
// log lines (DFAlign.cu:1124-1181).
static void sum_shifts(mc_plan* pl, std::vector<int>& frames, std::vector<cplx>& sh, std::vector<int>& apply) {
  const int nf = pl->nframe;
  int nss, nes, lim;
  sum_range(pl, &nss, &nes, &lim);
  pl->log("\nSum Frame #%03d - #%03d\n", nss + pl->nstart, nes + pl->nstart);
  cplx mid(0, 0);
  for (int j = 0; j < lim; j++) mid += pl->shift[j];
  cplx total(0, 0);
  for (int j = 1; j < nss + 1; j++) total += pl->shift[j - 1];
  frames.clear();
  sh.clear();
  apply.clear();
  pl->sum_shift.assign(nf, cplx(0, 0));
  for (int k = nss; k <= nes; k++) {
    if (k > nss) total += pl->shift[k - 1];
    const cplx s = -total + mid;
    frames.push_back(k);
    sh.push_back(s);
    apply.push_back((k == nss && !pl->p.bAlignToMid) ? 0 : 1);
    pl->sum_shift[k] = s;
    pl->log("......Add Frame #%03d with xy shift: %8.4lf %8.4lf\n", k + pl->nstart, s.real(), s.imag());
  }
  pl->sum_first = nss;
  pl->sum_last = nes;
  pl->have_sum = true;
}

extern "C" {

int mc_plan_sum(mc_plan* pl, float* image_host) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_iter) return set_err(MC_E_STATE, "sum before the shifts are final");
  CK(cudaSetDevice(pl->device));
  std::vector<int> frames, apply;
  std::vector<cplx> sh;
  sum_shifts(pl, frames, sh, apply);
  CK(cudaEventRecord(pl->ev[6], pl->st));
  CKR(run_shift_sum(pl, frames, sh, apply, 1));
  CK(cudaEventRecord(pl->ev[7], pl->st));
  if (image_host)
    CK(cudaMemcpyAsync(image_host, pl->d_image, sizeof(float) * (size_t)pl->n * pl->n, cudaMemcpyDeviceToHost,
                       pl->st));
  CK(cudaStreamSynchronize(pl->st));
  CK(cudaEventElapsedTime(&pl->tm.sum_ms, pl->ev[6], pl->ev[7]));
  CKR(pl->collect());
  return MC_OK;
}

// ------------------------------------------------- extra sum-stage outputs --
static int image_out(mc_plan* pl, float* image_host) {
  if (image_host)
    CK(cudaMemcpyAsync(image_host, pl->d_image, sizeof(float) * (size_t)pl->n * pl->n, cudaMemcpyDeviceToHost,
                       pl->st));
  CK(cudaStreamSynchronize(pl->st));
  return pl->collect();
}

int mc_plan_raw_sum(mc_plan* pl, float* image_host) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_forward) return set_err(MC_E_STATE, "raw sum before forward");
  CK(cudaSetDevice(pl->device));
  int nss, nes, lim;
  sum_range(pl, &nss, &nes, &lim);
  std::vector<int> frames, apply;
  std::vector<cplx> sh;
  for (int k = nss; k <= nes; k++) {
    frames.push_back(k);
    sh.push_back(cplx(0, 0));
    apply.push_back(0);
  }
  CKR(run_shift_sum(pl, frames, sh, apply, 1));
  return image_out(pl, image_host);
}

int mc_plan_sum_to(mc_plan* pl, int last_frame, float* image_host) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_sum) return set_err(MC_E_STATE, "second sum before the corrected sum");
  CK(cudaSetDevice(pl->device));
  // nEndSum2 clamps of DFAlign.cu:1117-1122
  int last = last_frame - pl->nstart;
  if (last <= pl->sum_first || last >= pl->nframe) last = pl->nframe - 1;
  if (last > pl->sum_last) last = pl->sum_last;
  std::vector<int> frames, apply;
  std::vector<cplx> sh;
  for (int k = pl->sum_first; k <= last; k++) {
    frames.push_back(k);
    sh.push_back(pl->sum_shift[k]);
    apply.push_back((k == pl->sum_first && !pl->p.bAlignToMid) ? 0 : 1);
  }
  CKR(run_shift_sum(pl, frames, sh, apply, 1));
  return image_out(pl, image_host);
}

int mc_plan_corrected_frame(mc_plan* pl, int frame, float* image_host) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_sum) return set_err(MC_E_STATE, "corrected frame before the corrected sum");
  const int k = frame - pl->nstart;
  if (k < pl->sum_first || k > pl->sum_last)
    return set_err(MC_E_ARG, "frame %d outside the summed range [%d, %d]", frame, pl->sum_first + pl->nstart,
                   pl->sum_last + pl->nstart);
  CK(cudaSetDevice(pl->device));
  const std::vector<int> frames{k};
  const std::vector<cplx> sh{pl->sum_shift[k]};
  const std::vector<int> apply{(k == pl->sum_first && !pl->p.bAlignToMid) ? 0 : 1};
  CKR(run_shift_sum(pl, frames, sh, apply, 1));
  return image_out(pl, image_host);
}

// Contrast mapping of the displays (histMinMax with a 0.5 % tail on each
// side over 400 bins, then buf2DispShort's linear map to 0..255;
// func.cpp:372-455), in the reference's float arithmetic.
static void display_short(const float* buf, int size, int16_t* disp) {
  float mn = 1e20f, mx = -1e20f;
  for (int i = 0; i < size; i++) {
    if (buf[i] < mn) mn = buf[i];
    if (buf[i] > mx) mx = buf[i];
  }
  std::fill(disp, disp + size, (int16_t)0);
  if (mn >= mx) return;
  const int nbin = 400;
  std::vector<int> hist(nbin, 0);
  const float step = (mx - mn) / nbin;
  for (int i = 0; i < size; i++) {
    int id = (int)((buf[i] - mn) / step);
    if (id >= nbin) id = nbin - 1;
    hist[id]++;
  }
  const int percent = (int)(size * 0.005f);
  int count = 0;
  for (int i = 0; i < nbin; i++) {
    count += hist[i];
    if (count > percent) {
      mn += i * step;
      break;
    }
  }
  count = 0;
  for (int i = nbin - 1; i > 0; i--) {
    count += hist[i];
    if (count > percent) {
      mx -= (nbin - 1 - i) * step;
      break;
    }
  }
  if (mn >= mx) return;
  const float scale = 255.0f / (mx - mn);
  for (int i = 0; i < size; i++) {
    if (buf[i] <= mn) disp[i] = 0;
    else if (buf[i] >= mx) disp[i] = 255;
    else disp[i] = (int16_t)((buf[i] - mn) * scale);
  }
}

// FSC of -fsc (PlotFSC, DFAlign.cu:212-326) over the corrected sum's frames.
int mc_plan_fsc(mc_plan* pl, double* rows, int cap, int* nbox_out) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_sum) return set_err(MC_E_STATE, "FSC before the corrected sum");
  if (pl->slots)
    return set_err(MC_E_STATE, "FSC reads every summed spectrum at once; this plan holds %d (spectrum slots)",
                   pl->slots);
  const int n = pl->n;
  if (n < 400) return set_err(MC_E_SIZE, "FSC needs nsam >= 400 (shell width nsam/400), nsam is %d", n);
  const int step = n / 400, nsamc = n / 2 + 1, nbox = nsamc / step + 1;
  if (nbox_out) *nbox_out = nbox;
  if (!rows) return MC_OK;  // size query
  CK(cudaSetDevice(pl->device));
  const int ns = pl->sum_last - pl->sum_first + 1;
  std::vector<int> frames(ns), apply(ns);
  std::vector<double2> sh(ns);
  for (int i = 0; i < ns; i++) {
    const int k = pl->sum_first + i;
    frames[i] = k;
    apply[i] = (k == pl->sum_first && !pl->p.bAlignToMid) ? 0 : 1;
    sh[i] = make_double2(pl->sum_shift[k].real(), pl->sum_shift[k].imag());
  }
  CK(cudaMemcpyAsync(pl->d_sumframes, frames.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, pl->st));
  CK(cudaMemcpyAsync(pl->d_apply, apply.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, pl->st));
  CK(cudaMemcpyAsync(pl->d_sumshift, sh.data(), sizeof(double2) * ns, cudaMemcpyHostToDevice, pl->st));
  const size_t nh = 12 * (size_t)nbox;
  if (!pl->d_fsc) {
    CKR(pl->alloc(&pl->d_fsc, sizeof(double) * nh * ((size_t)pl->H + 1)));
  }
  // direction: the drift of the last summed frame (totalshift, DFAlign.cu:1232-1234), unit length
  // when longer than 0.1 px, else the x axis (DFAlign.cu:235-236)
  cplx dir = pl->frame_shift.empty() ? cplx(0, 0) : pl->frame_shift[pl->sum_last];
  if (std::abs(dir) > 0.1) dir /= std::abs(dir);
  else dir = cplx(1.0, 0.0);
  mc::FscArgs a{};
  a.spec = pl->d_specA;
  a.stride = pl->fstride;
  a.frames = pl->d_sumframes;
  a.shifts = pl->d_sumshift;
  a.apply = pl->d_apply;
  a.nsum = ns;
  a.n = n;
  a.ldn = pl->ldn;
  a.H = pl->H;
  a.step = step;
  a.nbox = nbox;
  a.dirx = dir.real();
  a.diry = dir.imag();
  a.edge = (float)std::cos(M_PI / 4);
  a.part = pl->d_fsc + nh;
  a.out = pl->d_fsc;
  CK(mc::launch_fsc(a, pl->d_ey, pl->st));
  std::vector<double> t(nh);
  CK(cudaMemcpyAsync(t.data(), pl->d_fsc, sizeof(double) * nh, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  auto fsc = [](const double* v) {
    const double p = v[1] * v[2];
    return p > 0.00001 ? v[0] / std::sqrt(p) : 0.0;
  };
  for (int i = 0; i < nbox && i < cap; i++) {
    const double* d = t.data() + (size_t)i * 6;           // along the drift
    const double* u = t.data() + (size_t)(nbox + i) * 6;  // across it
    double* r = rows + (size_t)i * 5;
    r[0] = i * 100.0 / nbox;
    r[1] = fsc(d);
    r[2] = fsc(u);
    r[3] = fsc(d + 3);
    r[4] = fsc(u + 3);
  }
  return MC_OK;
}

int mc_plan_quicklook(mc_plan* pl, int which, int16_t* out) {
  constexpr int D = MC_QUICKLOOK_DIM;
  if (!pl || !out) return set_err(MC_E_ARG, "null argument");
  if (which < 0 || which > 2) return set_err(MC_E_ARG, "quick-look kind %d outside [0, 2]", which);
  const int n = pl->n;
  if (n < D) return set_err(MC_E_SIZE, "quick-look displays need a binned side of at least %d (got %d)", D, n);
  CK(cudaSetDevice(pl->device));
  // the sum spectrum into d_sum: unaligned (raw FFT) or corrected
  std::vector<int> frames, apply;
  std::vector<cplx> sh;
  if (which == 0) {
    if (!pl->have_forward) return set_err(MC_E_STATE, "quick-look before forward");
    int nss, nes, lim;
    sum_range(pl, &nss, &nes, &lim);
    for (int k = nss; k <= nes; k++) {
      frames.push_back(k);
      sh.push_back(cplx(0, 0));
      apply.push_back(0);
    }
  } else {
    if (!pl->have_sum) return set_err(MC_E_STATE, "quick-look of the corrected sum before the sum");
    for (int k = pl->sum_first; k <= pl->sum_last; k++) {
      frames.push_back(k);
      sh.push_back(pl->sum_shift[k]);
      apply.push_back((k == pl->sum_first && !pl->p.bAlignToMid) ? 0 : 1);
    }
  }
  CKR(run_shift_sum(pl, frames, sh, apply, 0));
  if (!pl->d_ql) {
    CKR(pl->alloc(&pl->d_ql, sizeof(float2) * 2 * (size_t)(D / 2 + 1) * D));
    CKR(pl->alloc(&pl->d_qlimg, sizeof(float) * (size_t)D * D));
  }
  float2* spec = pl->d_ql;
  float2* tmp = pl->d_ql + (size_t)(D / 2 + 1) * D;
  float scale = 1.0f;
  if (which == 1) {
    // GPUMemBinD2H + ifft2d of the sum (DFAlign.cu:1278-1282, 73-88)
    CK(mc::launch_ql_crop(pl->d_sum, pl->ldn, n, D, spec, pl->st));
  } else {
    // log modulus as the centred display image (cufunc.cu:178-188,
    // func.cpp:459-489), its R2C, Fourier crop to D, C2R / D^2
    // (BinFFTDispBufToChar, func.cpp:524-556)
    float* img = pl->d_image;
    CK(mc::launch_ql_logmod(pl->d_sum, pl->ldn, n, 1.0e-4f, img, pl->st));
    const int hk = D / 2 + 1;
    const int ldt = (int)round_up(n, 2);
    mc::FwdRowsArgs a{};
    a.frame = img;
    a.mode = 2;
    a.nx = n;
    a.ny = n;
    a.nu = n;
    a.hk = hk;
    a.outA = pl->d_T2;
    a.ldt = ldt;
    a.plan = pl->plan_n;
    a.tw = pl->d_tw_n;
    CK(mc::launch_fwd_rows(a, pl->st));
    mc::RowsFftArgs c{};
    c.in = pl->d_T2;
    c.ld_in = ldt;
    c.out = spec;
    c.ld_out = D;
    c.nrows = hk;
    c.n_out = D;
    c.keep_lo = D / 2;
    c.scale = 1.f;
    c.plan = pl->plan_n;
    c.tw = pl->d_tw_n;
    CK(mc::launch_rows_fft(c, false, 1, pl->st));
    scale = 1.0f / ((float)D * D);
  }
  CK(mc::launch_ql_c2r(spec, D, scale, tmp, pl->d_qlimg, pl->st));
  std::vector<float> h((size_t)D * D);
  CK(cudaMemcpyAsync(h.data(), pl->d_qlimg, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  CKR(pl->collect());
  display_short(h.data(), D * D, out);
  return MC_OK;
}

int mc_plan_count_sum(mc_plan* pl, int32_t* host) {
  if (!pl || !host) return set_err(MC_E_ARG, "null argument");
  if (pl->mode == 2 || pl->mode == MC_MODE_F16)
    return set_err(MC_E_ARG, "count sums need integer pixels (mode 0, 1, 6 or MC_MODE_U8)");
  for (int f = 0; f < pl->nframe; f++)
    if (!pl->loaded[f]) return set_err(MC_E_STATE, "frame position %d not loaded", f);
  CK(cudaSetDevice(pl->device));
  if (!pl->d_count) CKR(pl->alloc(&pl->d_count, sizeof(int) * (size_t)pl->nu * pl->nu));
  int nss, nes, lim;
  sum_range(pl, &nss, &nes, &lim);
  mc::CountSumArgs a{};
  a.frames = pl->frames_src ? pl->frames_src : pl->d_frames;
  a.frame_pixels = (long long)pl->nx * pl->ny;
  a.mode = pl->mode;
  a.nx = pl->nx;
  a.offx = pl->p.crop_offsetx;
  a.offy = pl->p.crop_offsety;
  a.nu = pl->nu;
  a.first = nss;
  a.last = nes;
  a.out = pl->d_count;
  CK(mc::launch_count_sum(a, pl->st));
  CK(cudaMemcpyAsync(host, pl->d_count, sizeof(int) * (size_t)pl->nu * pl->nu, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  return MC_OK;
}

// Objective of the gradient refinement at sum shifts s (2*nframe): J, its
// gradient (2*nframe) and the 2x2 Hessian blocks (3*nframe: xx, xy, yy).
// Pass 1 is the phase-shift-and-sum into d_sum, pass 2 the adjoint kernel.
static int objective(mc_plan* pl, const std::vector<cplx>& s, double* J, double* grad, double* hess) {
  const int nf = pl->nframe;
  std::vector<int> frames(nf), apply(nf, 1);
  for (int k = 0; k < nf; k++) frames[k] = k;
  CKR(run_shift_sum(pl, frames, s, apply, 0));  // also leaves the ky ramps of s in d_ey
  mc::ObjectiveArgs a{};
  a.spec = pl->d_specA;
  a.stride = pl->fstride;
  a.nframes = nf;
  a.S = pl->d_sum;
  a.shifts = pl->d_sumshift;
  a.ey = pl->d_ey;
  a.n = pl->n;
  a.ldn = pl->ldn;
  a.H = pl->H;
  a.mbf = (float)(-0.5 * (double)pl->p.bfactor / pl->n / pl->n);
  a.partial = pl->d_opart;
  a.partialJ = pl->d_opart + (size_t)pl->H * nf * 5;
  a.out = pl->d_oout;
  if (pl->slots) {
    // slot mode: the adjoint pass over chunks of `slots` frames (their
    // spectra held again, their shifts and ramps re-laid), each chunk's
    // per-frame totals at its frames' places; every chunk also writes J at
    // the entry after its last frame, which the next chunk overwrites, so the
    // last chunk's J (the same sum over S each time) is the one left
    for (int c0 = 0; c0 < nf; c0 += pl->slots) {
      const int cnt = std::min(pl->slots, nf - c0);
      const std::vector<int> fr(frames.begin() + c0, frames.begin() + c0 + cnt);
      std::vector<int> where;
      CKR(hold_spectra(pl, fr, where));
      std::vector<double2> sh(cnt);
      for (int i = 0; i < cnt; i++) sh[i] = make_double2(s[c0 + i].real(), s[c0 + i].imag());
      CK(cudaMemcpyAsync(pl->d_sumframes, where.data(), sizeof(int) * cnt, cudaMemcpyHostToDevice, pl->st));
      CK(cudaMemcpyAsync(pl->d_sumshift, sh.data(), sizeof(double2) * cnt, cudaMemcpyHostToDevice, pl->st));
      CK(mc::launch_ramp(pl->d_sumshift, cnt, pl->n, pl->d_ey, pl->st));
      mc::ObjectiveArgs b = a;
      b.frames = pl->d_sumframes;
      b.nframes = cnt;
      b.partialJ = pl->d_opart + (size_t)pl->H * cnt * 5;
      b.out = pl->d_oout + (size_t)c0 * 5;
      LAUNCH_N(pl, MC_K_OBJECTIVE, (double)(cnt + 1) * pl->H * pl->n * sizeof(float2), 2,
               mc::launch_objective(b, pl->st));
    }
  } else {
    LAUNCH_N(pl, MC_K_OBJECTIVE, (double)(nf + 1) * pl->H * pl->n * sizeof(float2), 2,
             mc::launch_objective(a, pl->st));
  }
  std::vector<double> out((size_t)nf * 5 + 1);
  CK(cudaMemcpyAsync(out.data(), pl->d_oout, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  CKR(pl->collect());
  if (J) *J = out[(size_t)nf * 5];
  for (int k = 0; k < nf; k++) {
    if (grad) {
      grad[2 * k] = out[5 * k];
      grad[2 * k + 1] = out[5 * k + 1];
    }
    if (hess) {
      hess[3 * k] = out[5 * k + 2];
      hess[3 * k + 1] = out[5 * k + 3];
      hess[3 * k + 2] = out[5 * k + 4];
    }
  }
  return MC_OK;
}

int mc_plan_objective(mc_plan* pl, const double* shifts_xy, double* J, double* grad, double* hess) {
  if (!pl || !shifts_xy) return set_err(MC_E_ARG, "null argument");
  if (!pl->have_forward) return set_err(MC_E_STATE, "objective before forward");
  CK(cudaSetDevice(pl->device));
  std::vector<cplx> s(pl->nframe);
  for (int k = 0; k < pl->nframe; k++) s[k] = cplx(shifts_xy[2 * k], shifts_xy[2 * k + 1]);
  return objective(pl, s, J, grad, hess);
}

// Block-Newton ascent of J over every frame's sum shift, starting from the
// peak-fit solution; frame 0 stays the reference of the refined shifts.
int mc_plan_refine(mc_plan* pl, int iterations) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_iter) return set_err(MC_E_STATE, "refine before the peak-fit shifts are final");
  CK(cudaSetDevice(pl->device));
  const int nf = pl->nframe;
  std::vector<cplx> s(nf);
  for (int k = 0; k < nf; k++) s[k] = -pl->frame_shift[k];
  std::vector<double> g(2 * (size_t)nf), h(3 * (size_t)nf);
  double J = 0.0, maxd = 0.0;
  int it;
  CK(cudaEventRecord(pl->ev[4], pl->st));
  for (it = 0; it < iterations; it++) {
    CKR(objective(pl, s, &J, g.data(), h.data()));
    maxd = 0.0;
    for (int k = 0; k < nf; k++) {
      const double a = h[3 * k], b = h[3 * k + 1], c = h[3 * k + 2];
      const double det = a * c - b * b;
      if (!(a < 0.0 && det > 0.0)) continue;  // not at a local maximum in this frame: leave it
      double dx = -(c * g[2 * k] - b * g[2 * k + 1]) / det;
      double dy = -(-b * g[2 * k] + a * g[2 * k + 1]) / det;
      const double len = std::sqrt(dx * dx + dy * dy);
      if (len > 0.25) {  // trust region of a quarter pixel per step
        dx *= 0.25 / len;
        dy *= 0.25 / len;
      }
      s[k] += cplx(dx, dy);
      maxd = std::max(maxd, std::sqrt(dx * dx + dy * dy));
    }
    if (maxd < 1e-4) {
      it++;
      break;
    }
  }
  CK(cudaEventRecord(pl->ev[5], pl->st));
  CK(cudaEventSynchronize(pl->ev[5]));
  CK(cudaEventElapsedTime(&pl->tm.refine_ms, pl->ev[4], pl->ev[5]));
  for (int k = 0; k < nf; k++) pl->frame_shift[k] = s[0] - s[k];
  for (int k = 0; k < nf - 1; k++) pl->shift[k] = pl->frame_shift[k + 1] - pl->frame_shift[k];
  pl->have_sum = false;
  pl->log("\nGradient refinement: %d Newton step(s), last max update %.5f px, objective %.6e\n", it, maxd, J);
  for (int k = 0; k < nf; k++)
    pl->log("......Refined shift of Frame #%03d : %8.4f %8.4f\n", k + pl->nstart, pl->frame_shift[k].real(),
            pl->frame_shift[k].imag());
  return MC_OK;
}

}  // extern "C"

// pairs -> device solve -> sum -> result copies into the pinned staging,
// all on the plan stream without a host synchronisation.
static int enqueue_tail(mc_plan* pl, unsigned char* hs) {
  const int np = (int)pl->pairs.size(), nf = pl->nframe, nc = nf - 1;
  CK(cudaMemcpy2DAsync(hs + pl->st_dc, sizeof(float2), pl->d_specA, sizeof(float2) * pl->fstride, sizeof(float2),
                       nf, cudaMemcpyDeviceToHost, pl->st));
  CKR(enqueue_pair_stage(pl, pl->d_specA, pl->fstride, pl->d_specB, pl->fstride, pl->pairs, pl->d_pairs_main));
  int nss, nes, lim;
  sum_range(pl, &nss, &nes, &lim);
  mc::SolveArgs s{};
  s.pairs = pl->d_pairs_main;
  s.npairs = np;
  s.pshift = pl->d_pshift;
  s.nframe = nf;
  s.kithresh = pl->p.kiThresh;
  s.align_to_mid = pl->p.bAlignToMid ? 1 : 0;
  s.mid_steps = lim;
  s.sum_first = nss;
  s.sum_last = nes;
  s.M = pl->d_M;
  s.rhs = pl->d_rhs;
  s.work = pl->d_work;
  s.mask = pl->d_mask;
  s.order = pl->d_order;
  s.uf = pl->d_uf;
  s.ki1 = pl->d_ki1;
  s.kept = pl->d_kept;
  s.nkept = pl->d_nkept;
  s.ki2 = pl->d_ki2;
  s.shift = pl->d_dshift;
  s.frame_shift = pl->d_dfshift;
  s.sum_shift = pl->d_sumshift;
  s.sum_frames = pl->d_sumframes;
  s.sum_apply = pl->d_apply;
  s.status = pl->d_status;
  LAUNCH(pl, MC_K_SOLVE, (double)np * (2 * sizeof(float) + 2 * sizeof(double) + sizeof(int)) + (double)nf * 4 * sizeof(double),
         mc::launch_solve(s, pl->st));
  mc::ShiftSumArgs a{};
  a.spec = pl->d_specA;
  a.stride = pl->fstride;
  a.frames = pl->d_sumframes;
  a.shifts = pl->d_sumshift;
  a.apply = pl->d_apply;
  a.nsum = nes - nss + 1;
  a.n = pl->n;
  a.ldn = pl->ldn;
  a.H = pl->H;
  a.mode = 1;
  a.plan = pl->plan_n;
  a.tw = pl->d_tw_n;
  a.acc = pl->d_sumacc;
  a.out = pl->d_T2;
  a.ld_out = pl->ldt2;
  const double spec_bytes = (double)pl->H * pl->n * sizeof(float2);
  LAUNCH_N(pl, MC_K_SHIFT_SUM, (double)a.nsum * spec_bytes + spec_bytes, mc::shift_sum_kernels(a),
           mc::launch_shift_sum(a, pl->d_ey, pl->st));
  mc::C2rRowsArgs c{};
  c.t2 = pl->d_T2;
  c.ld_t2 = pl->ldt2;
  c.n = pl->n;
  c.H = pl->H;
  c.scale = (float)(1.0 / ((double)pl->n * pl->n));
  c.image = pl->d_image;
  c.plan = pl->plan_n;
  c.tw = pl->d_tw_n;
  LAUNCH(pl, MC_K_C2R_ROWS, spec_bytes + (double)pl->n * pl->n * sizeof(float), mc::launch_c2r_rows(c, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_pshift, pl->d_pshift, sizeof(float) * 2 * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_pcc, pl->d_pcc, sizeof(float) * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_ppeak, pl->d_ppeak, sizeof(int) * 2 * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_ki1, pl->d_ki1, sizeof(double) * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_kept, pl->d_kept, sizeof(int) * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_nkept, pl->d_nkept, sizeof(int), cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_ki2, pl->d_ki2, sizeof(double) * np, cudaMemcpyDeviceToHost, pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_work, pl->d_work, sizeof(double) * 2 * (size_t)nc, cudaMemcpyDeviceToHost,
                     pl->st));
  CK(cudaMemcpyAsync(hs + pl->st_status, pl->d_status, sizeof(int), cudaMemcpyDeviceToHost, pl->st));
  return MC_OK;
}

// After the stream synchronised: results into the plan's host state, with the
// same log lines as the staged path.
static int finish_device_movie(mc_plan* pl, const unsigned char* hs) {
  const int np = (int)pl->pairs.size(), nc = pl->nframe - 1;
  if (*(const int*)(hs + pl->st_status) != 0) return set_err(MC_E_NUMERIC, "singular pair system");
  log_frame_means(pl, (const float2*)(hs + pl->st_dc));
  pl->have_forward = true;
  const float* ps = (const float*)(hs + pl->st_pshift);
  pl->pshift.assign(ps, ps + 2 * (size_t)np);
  const float* pc = (const float*)(hs + pl->st_pcc);
  pl->pcc.assign(pc, pc + np);
  const int* pk = (const int*)(hs + pl->st_ppeak);
  pl->ppeak.assign(pk, pk + 2 * (size_t)np);
  log_pairs(pl);
  pl->have_pairs = true;
  const double* k1 = (const double*)(hs + pl->st_ki1);
  pl->ki1.assign(k1, k1 + np);
  const int nk = *(const int*)(hs + pl->st_nkept);
  const int* kp = (const int*)(hs + pl->st_kept);
  pl->good.assign(kp, kp + nk);
  const double* k2 = (const double*)(hs + pl->st_ki2);
  pl->ki2.assign(k2, k2 + nk);
  log_solve(pl);
  const double* w = (const double*)(hs + pl->st_work);
  pl->shift.resize(nc);
  for (int k = 0; k < nc; k++) pl->shift[k] = cplx(w[k], w[nc + k]);
  pl->have_solve = true;
  CKR(mc_plan_iterate(pl));  // itr = 0: the reference's conversions and log lines only
  std::vector<int> frames, apply;
  std::vector<cplx> sh;
  sum_shifts(pl, frames, sh, apply);
  return MC_OK;
}

// Whole movie on the device with one synchronisation; captured once into a
// CUDA graph and replayed (unless profiling or a capture failure).
static int run_device(mc_plan* pl, float* image_host, const std::vector<cudaEvent_t>* waits, int chunk) {
  const bool graph_ok = !waits && !pl->profiling && !pl->graph_failed;
  CKR(upload_frame_base(pl));
  CK(cudaEventRecord(pl->ev[0], pl->st));
  mc_plan::GraphEntry* ge = nullptr;
  if (graph_ok) {
    int nss, nes, lim;
    sum_range(pl, &nss, &nes, &lim);
    long long kt;
    float kf = pl->p.kiThresh;
    std::memcpy(&kt, &kf, sizeof(float));
    const std::vector<long long> key = {pl->nstart, pl->nend, nss, nes, lim, pl->p.FrameDistOffset,
                                        pl->p.bAlignToMid ? 1 : 0, kt & 0xffffffffLL,
                                        };
    for (auto& g : pl->graphs)
      if (g.key == key) ge = &g;
    if (!ge) {
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(pl->st, cudaStreamCaptureModeThreadLocal));
      pl->capturing = true;
      for (int k = 0; k < MC_KERNEL_KINDS; k++) {
        pl->graph_kcount[k] = 0;
        pl->graph_kbytes[k] = 0;
      }
      int rc = enqueue_forward(pl, nullptr, 1);
      if (rc == MC_OK) rc = enqueue_tail(pl, pl->h_stage);
      pl->capturing = false;
      const cudaError_t e = cudaStreamEndCapture(pl->st, &g);
      cudaGetLastError();
      cudaGraphExec_t x = nullptr;
      if (rc == MC_OK && e == cudaSuccess && g && cudaGraphInstantiate(&x, g, 0) == cudaSuccess) {
        cudaGraphDestroy(g);
        if (pl->graphs.size() >= 16) {  // keep the cache bounded: drop the oldest
          cudaGraphExecDestroy(pl->graphs.front().exec);
          pl->graphs.erase(pl->graphs.begin());
        }
        mc_plan::GraphEntry n;
        n.key = key;
        n.exec = x;
        std::copy(pl->graph_kcount, pl->graph_kcount + MC_KERNEL_KINDS, n.kcount);
        std::copy(pl->graph_kbytes, pl->graph_kbytes + MC_KERNEL_KINDS, n.kbytes);
        pl->graphs.push_back(n);
        ge = &pl->graphs.back();
      } else {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        pl->graph_failed = true;
      }
    }
  }
  if (ge) {
    CK(cudaGraphLaunch(ge->exec, pl->st));
    for (int k = 0; k < MC_KERNEL_KINDS; k++) {
      pl->kcount[k] += ge->kcount[k];
      pl->kbytes[k] += ge->kbytes[k];
    }
  } else {
    CKR(enqueue_forward(pl, waits, chunk));
    CKR(enqueue_tail(pl, pl->h_stage));
  }
  CK(cudaEventRecord(pl->ev[1], pl->st));
  if (image_host)
    CK(cudaMemcpyAsync(image_host, pl->d_image, sizeof(float) * (size_t)pl->n * pl->n, cudaMemcpyDeviceToHost,
                       pl->st));
  CK(cudaStreamSynchronize(pl->st));
  CKR(pl->collect());
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, pl->ev[0], pl->ev[1]));
  pl->tm = mc_timings{};
  pl->tm.total_ms = ms;
  return finish_device_movie(pl, pl->h_stage);
}

static bool device_path(const mc_plan* pl) { return pl->p.iter == 0 && !pl->p.refine && !pl->slots; }

extern "C" {

int mc_plan_run(mc_plan* pl, float* image_host) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  pl->log("Input Stack: Nx(%d) Ny(%d) Nz(%d) Mode(%d)\n\n", pl->nx, pl->ny, pl->nz, pl->mode);
  pl->log("Crop Image: Offset(%d %d) RawDim(%d) BinnedDim(%d)\n", pl->p.crop_offsetx, pl->p.crop_offsety, pl->nu,
          pl->n);
  if (device_path(pl)) {
    for (int f = 0; f < pl->nframe; f++)
      if (!pl->loaded[f]) return set_err(MC_E_STATE, "frame position %d not loaded", f);
    CK(cudaSetDevice(pl->device));
    return run_device(pl, image_host, nullptr, 1);
  }
  CKR(mc_plan_forward(pl));
  CKR(mc_plan_pairs(pl));
  CKR(mc_plan_solve(pl));
  CKR(mc_plan_iterate(pl));
  pl->tm.refine_ms = 0.f;
  if (pl->p.refine) CKR(mc_plan_refine(pl, 4));
  CKR(mc_plan_sum(pl, image_host));
  pl->tm.total_ms = pl->tm.forward_ms + pl->tm.pairs_ms + pl->tm.iterate_ms + pl->tm.refine_ms + pl->tm.sum_ms;
  return MC_OK;
}

int mc_plan_get_frame_shifts(const mc_plan* pl, double* xy) {
  if (!pl || !xy) return set_err(MC_E_ARG, "null argument");
  if (!pl->have_iter) return set_err(MC_E_STATE, "no final shifts yet");
  for (int k = 0; k < pl->nframe; k++) {
    xy[2 * k] = pl->frame_shift[k].real();
    xy[2 * k + 1] = pl->frame_shift[k].imag();
  }
  return MC_OK;
}

int mc_plan_get_pairs(const mc_plan* pl, int* ij, float* shift, float* cc, int* peak) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_pairs) return set_err(MC_E_STATE, "no pair results yet");
  const size_t np = pl->pairs.size();
  for (size_t j = 0; j < np; j++) {
    if (ij) {
      ij[2 * j] = pl->pairs[j].first;
      ij[2 * j + 1] = pl->pairs[j].second;
    }
    if (shift) {
      shift[2 * j] = pl->pshift[2 * j];
      shift[2 * j + 1] = pl->pshift[2 * j + 1];
    }
    if (cc) cc[j] = pl->pcc[j];
    if (peak) {
      peak[2 * j] = pl->ppeak[2 * j];
      peak[2 * j + 1] = pl->ppeak[2 * j + 1];
    }
  }
  return MC_OK;
}

int mc_plan_get_ki(const mc_plan* pl, double* ki1, int* nkept, int* kept, double* ki2) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (!pl->have_solve) return set_err(MC_E_STATE, "no solve yet");
  if (ki1) std::copy(pl->ki1.begin(), pl->ki1.end(), ki1);
  if (nkept) *nkept = (int)pl->good.size();
  if (kept) std::copy(pl->good.begin(), pl->good.end(), kept);
  if (ki2) std::copy(pl->ki2.begin(), pl->ki2.end(), ki2);
  return MC_OK;
}

int mc_plan_get_frame_means(const mc_plan* pl, float* mean) {
  if (!pl || !mean) return set_err(MC_E_ARG, "null argument");
  if (!pl->have_forward) return set_err(MC_E_STATE, "no forward yet");
  std::copy(pl->frame_mean.begin(), pl->frame_mean.end(), mean);
  return MC_OK;
}

int mc_plan_get_spectrum(mc_plan* pl, int set, int pos, void* host) {
  if (!pl || !host) return set_err(MC_E_ARG, "null argument");
  if (!pl->have_forward) return set_err(MC_E_STATE, "no forward yet");
  if (pos < 0 || pos >= pl->nframe || set < 0 || set > 1) return set_err(MC_E_ARG, "bad set/pos");
  CK(cudaSetDevice(pl->device));
  std::vector<int> where;
  CKR(hold_spectra(pl, {pos}, where));
  const float2* src = (set == 0 ? pl->d_specA : pl->d_specB) + (long long)where[0] * pl->fstride;
  CK(cudaMemcpy2DAsync(host, sizeof(float2) * pl->n, src, sizeof(float2) * pl->ldn, sizeof(float2) * pl->n, pl->H,
                       cudaMemcpyDeviceToHost, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  return MC_OK;
}

int mc_plan_get_boxes(mc_plan* pl, float* host) {
  if (!pl || !host) return set_err(MC_E_ARG, "null argument");
  if (!pl->have_pairs) return set_err(MC_E_STATE, "no pair results yet");
  CK(cudaSetDevice(pl->device));
  CK(cudaMemcpyAsync(host, pl->d_boxes, sizeof(float) * pl->pairs.size() * pl->box * pl->box,
                     cudaMemcpyDeviceToHost, pl->st));
  CK(cudaStreamSynchronize(pl->st));
  return MC_OK;
}

int mc_plan_get_sum_shifts(const mc_plan* pl, double* xy, int* first, int* last) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  if (xy)
    for (int k = 0; k < pl->nframe; k++) {
      xy[2 * k] = k < (int)pl->sum_shift.size() ? pl->sum_shift[k].real() : 0.0;
      xy[2 * k + 1] = k < (int)pl->sum_shift.size() ? pl->sum_shift[k].imag() : 0.0;
    }
  if (first) *first = pl->sum_first;
  if (last) *last = pl->sum_last;
  return MC_OK;
}

int mc_plan_get_timings(const mc_plan* pl, mc_timings* t) {
  if (!pl || !t) return set_err(MC_E_ARG, "null argument");
  *t = pl->tm;
  return MC_OK;
}

void mc_plan_set_profiling(mc_plan* pl, int on) {
  if (pl) pl->profiling = on != 0;
}

int mc_plan_reset_stats(mc_plan* pl) {
  if (!pl) return set_err(MC_E_ARG, "null plan");
  for (int k = 0; k < MC_KERNEL_KINDS; k++) {
    pl->kms[k] = 0;
    pl->kbytes[k] = 0;
    pl->kcount[k] = 0;
  }
  return MC_OK;
}

int mc_plan_kernel_stats(const mc_plan* pl, int kind, double* ms, long long* launches, double* bytes) {
  if (!pl || kind < 0 || kind >= MC_KERNEL_KINDS) return set_err(MC_E_ARG, "bad kernel kind");
  if (ms) *ms = pl->kms[kind];
  if (launches) *launches = pl->kcount[kind];
  if (bytes) *bytes = pl->kbytes[kind];
  return MC_OK;
}

const char* mc_kernel_name(int kind) {
  static const char* names[MC_KERNEL_KINDS] = {"k_fwd_rows", "k_rows_fft", "k_pair_cols", "k_pair_rows",
                                               "k_peak", "k_shift_sum", "k_c2r_rows", "k_objective",
                                               "k_solve"};
  return (kind >= 0 && kind < MC_KERNEL_KINDS) ? names[kind] : "";
}

int mc_solve_pairs(int nframe, int npairs, const int* ij, const float* shifts_xy, float kithresh,
                   double* step_xy, double* ki1, int* nkept, int* kept, double* ki2) {
  if (nframe < 2 || npairs < 1 || !ij || !shifts_xy) return set_err(MC_E_ARG, "bad solve arguments");
  std::vector<mc::PairIJ> rows(npairs);
  std::vector<cplx> b(npairs);
  std::vector<int> all(npairs);
  for (int r = 0; r < npairs; r++) {
    const int i = ij[2 * r], j = ij[2 * r + 1];
    if (i < 0 || j <= i || j >= nframe) return set_err(MC_E_ARG, "pair %d (%d, %d) invalid", r, i, j);
    rows[r] = {i, j};
    b[r] = cplx(shifts_xy[2 * r], shifts_xy[2 * r + 1]);
    all[r] = r;
  }
  std::vector<cplx> s;
  if (!mc::lsq_intervals(rows, all, nframe - 1, b, s)) return set_err(MC_E_NUMERIC, "singular pair system");
  const std::vector<double> k1 = mc::lsq_residuals(rows, all, b, s);
  const std::vector<int> good = mc::od_threshold(rows, k1, nframe, (double)kithresh);
  if (!mc::lsq_intervals(rows, good, nframe - 1, b, s)) return set_err(MC_E_NUMERIC, "singular pair system");
  const std::vector<double> k2 = mc::lsq_residuals(rows, good, b, s);
  if (step_xy)
    for (int k = 0; k < nframe - 1; k++) {
      step_xy[2 * k] = s[k].real();
      step_xy[2 * k + 1] = s[k].imag();
    }
  if (ki1) std::copy(k1.begin(), k1.end(), ki1);
  if (nkept) *nkept = (int)good.size();
  if (kept) std::copy(good.begin(), good.end(), kept);
  if (ki2) std::copy(k2.begin(), k2.end(), ki2);
  return MC_OK;
}

int mc_fft1d(int n, int batch, int inverse, const void* d_in, void* d_out, void* stream) {
  if (n < 1 || batch < 1 || !d_in || !d_out) return set_err(MC_E_ARG, "bad fft arguments");
  if ((size_t)3 * n * sizeof(float2) > 227 * 1024) return set_err(MC_E_SIZE, "n=%d too large", n);
  FftPlan1D p{};
  if (!make_plan(n, p)) return set_err(MC_E_SIZE, "no FFT plan for %d", n);
  float2* tw = nullptr;
  CK(cudaMalloc(&tw, sizeof(float2) * n));
  std::vector<float2> t = twiddles(n, -1);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(tw, t.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    mc::RowsFftArgs a{};
    a.in = (const float2*)d_in;
    a.ld_in = n;
    a.out = (float2*)d_out;
    a.ld_out = n;
    a.nrows = batch;
    a.n_out = n;
    a.keep_lo = n;
    a.scale = 1.f;
    a.plan = p;
    a.tw = tw;
    e = mc::launch_rows_fft(a, inverse != 0, 1, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(tw);
  if (e != cudaSuccess) return set_err(MC_E_CUDA, "mc_fft1d: %s", cudaGetErrorString(e));
  return MC_OK;
}

}  // extern "C"

// ------------------------------------------- batch captured as one graph --
// (mc_internal.h; used by mc_batch.cpp)
size_t mc::plan_stage_bytes(const mc_plan* pl) { return pl->st_bytes; }

bool mc::plan_device_only(const mc_plan* pl) { return device_path(pl) && !pl->two_sets && !pl->stretch; }

cudaStream_t mc::plan_stream(const mc_plan* pl) { return pl->st; }

int mc::plan_reframe_host(mc_plan* pl, const mc_params* p, int nz) {
  if (!pl || !p) return set_err(MC_E_ARG, "null argument");
  if (nz <= 1) return set_err(MC_E_ARG, "Not a stack or wrong file. Abort");
  pl->p.iter = p->iter;
  pl->p.iterthres = p->iterthres;
  pl->p.refine = p->refine;
  return configure_frames(pl, *p, nz, false);
}

int mc::plan_pair_words(const mc_plan* pl, int* ij, int cap) {
  const int np = (int)pl->pairs.size();
  if (np > cap) return set_err(MC_E_STATE, "pair list larger than its block");
  for (int j = 0; j < np; j++) {
    ij[2 * j] = pl->pairs[j].first;
    ij[2 * j + 1] = pl->pairs[j].second;
  }
  return MC_OK;
}

int mc::plan_enqueue_movie(mc_plan* pl, const void* const* frame_word, const int* pairs, unsigned char* stage,
                           float* image) {
  if (!device_path(pl))
    return set_err(MC_E_STATE, "movie is not device-only (-itr 0, no refinement, every spectrum resident)");
  CK(cudaMemcpyAsync(pl->d_pairs_main, pairs, sizeof(int2) * pl->pairs.size(), cudaMemcpyHostToDevice, pl->st));
  CK(cudaMemcpyAsync(pl->d_src_slot, frame_word, sizeof(void*), cudaMemcpyHostToDevice, pl->st));
  pl->capturing = true;
  int rc = enqueue_forward(pl, nullptr, 1);
  if (rc == MC_OK) rc = enqueue_tail(pl, stage);
  pl->capturing = false;
  CKR(rc);
  if (image)
    CK(cudaMemcpyAsync(image, pl->d_image, sizeof(float) * (size_t)pl->n * pl->n, cudaMemcpyDefault, pl->st));
  return MC_OK;
}

int mc::plan_finish_movie(mc_plan* pl, const unsigned char* stage, const void* d_frames) {
  pl->frames_src = d_frames;
  pl->loaded.assign(pl->nframe, 1);
  pl->tm = mc_timings{};
  return finish_device_movie(pl, stage);
}
