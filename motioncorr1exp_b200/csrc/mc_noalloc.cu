// Cross-correlation window of one frame pair without any device allocation.
//
// Some callers cannot call cudaMalloc: code that runs inside a detector's
// acquisition or streaming loop with a fixed, pre-reserved device-memory
// budget (an allocation there can block the loop or fail under memory
// pressure), and host frameworks that forbid allocation once their own
// memory pool is set up.  For them mc_pair_window_static() computes the
// pbx x pbx CC window of one frame pair that a plan's pair stage computes
// (the reference's GPUShiftCC + GPUIFFT2d + the FindShift box copy,
// cufunc.cu:343-407) for two spectra the caller already holds, with the same
// column kernel and split as the plan, using only the file-scope scratch
// array below for its intermediate data.
//
// Limits: n even, 16 <= n <= 4096, 16 <= pbx <= min(128, n), and n must split
// as n = P*Q with P <= 128 and Q one of the register-codelet lengths.  The
// scratch is kNoAllocScratchBytes (5 MiB) of device memory that every GPU
// which loads libmc holds until the process exits.
//
// The first call on a device resolves the array's device address there
// (cudaGetSymbolAddress with that device current) and remembers it; make that
// first call before any stream capture.  Every call on a device shares the
// same array and leaves its contents behind; calls whose work overlaps on the
// GPU (different streams, different host threads) race on it, so callers must
// serialise them.  Nothing in the scratch has to start at zero: every table
// and every intermediate element is fully written before it is read.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/mc.h"
#include "kernels.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)5 << 20;
constexpr int kNoAllocMaxN = 4096;
constexpr int kNoAllocMaxBox = 128;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// the text is reported by mc_last_error()
int fail(int code, const char* text) { return mc::record_error(code, text); }

// Device address of the scratch array on the current device (resolved once).
int scratch_on_current_device(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(MC_E_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return fail(MC_E_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return fail(MC_E_CUDA, "cudaGetSymbolAddress(scratch) failed");
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return MC_OK;
}

// Tables of the column and row stages, written into the scratch on device:
//   two[k1][m] = exp(+2 pi i k1 y_m / n),  y_m = (ystart + m) mod n
//   cs[kx][m]  = h(kx) exp(+2 pi i kx x_m / n), h = 1 at kx = 0, n/2 else 2
__global__ void k_noalloc_tables(float2* two, float2* cs, int2* pair, int n, int box, int P, int H, int ystart) {
  const int total = P * box + H * box;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const bool outer = t < P * box;
    const int u = outer ? t : t - P * box;
    const int k = u / box, m = u - k * box;
    const long long y = (ystart + m) % n;
    const long long e = ((long long)k * y) % n;
    double sn, cn;
    sincospi(2.0 * (double)e / (double)n, &sn, &cn);
    if (outer) {
      two[u] = make_float2((float)cn, (float)sn);
    } else {
      const double h = (k == 0 || k == n / 2) ? 1.0 : 2.0;
      cs[u] = make_float2((float)(h * cn), (float)(h * sn));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *pair = make_int2(0, 0);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

int mc_pair_window_static(const void* d_spec_a, const void* d_spec_b, int n, int ldn, int pbx, float bfactor,
                          float* d_window, void* stream) {
  if (!d_spec_a || !d_spec_b || !d_window) return fail(MC_E_ARG, "null pointer");
  if (n < 16 || n > kNoAllocMaxN || (n & 1)) return fail(MC_E_SIZE, "n must be even and in [16, 4096]");
  if (ldn < n) return fail(MC_E_ARG, "ldn < n");
  if (pbx < 16 || pbx > kNoAllocMaxBox || pbx > n) return fail(MC_E_SIZE, "pbx must be in [16, min(128, n)]");
  int P = 0, Q = 0;
  if (!mc::reg_pair_split(n, pbx, &P, &Q)) return fail(MC_E_SIZE, "n has no register-codelet split");
  const int H = n / 2 + 1;
  const size_t off_two = 256;  // the int2 pair record sits at the start
  const size_t off_cs = off_two + align256(sizeof(float2) * (size_t)P * pbx);
  const size_t off_g = off_cs + align256(sizeof(float2) * (size_t)H * pbx);
  const size_t need = off_g + align256(sizeof(float2) * (size_t)H * pbx);
  if (need > kNoAllocScratchBytes) return fail(MC_E_SIZE, "problem larger than the static scratch");
  void* base = nullptr;
  const int rc = scratch_on_current_device(&base);
  if (rc != MC_OK) return rc;
  unsigned char* s = (unsigned char*)base;
  int2* pair = (int2*)s;
  float2* two = (float2*)(s + off_two);
  float2* cs = (float2*)(s + off_cs);
  float2* G = (float2*)(s + off_g);
  cudaStream_t st = (cudaStream_t)stream;
  const int ori = (n - pbx) / 2;
  const int ystart = (ori + n / 2) % n;
  // an error left by an earlier, unrelated launch must not be reported as
  // this call's failure
  (void)cudaGetLastError();
  k_noalloc_tables<<<64, 256, 0, st>>>(two, cs, pair, n, pbx, P, H, ystart);
  if (cudaGetLastError() != cudaSuccess) return fail(MC_E_CUDA, "table kernel launch failed");
  mc::PairColsArgs a{};
  a.specA = (const float2*)d_spec_a;
  a.strideA = 0;
  a.specB = (const float2*)d_spec_b;
  a.strideB = 0;
  a.pairs = pair;
  a.npairs = 1;
  a.pairs_per_cta = 1;
  a.n = n;
  a.ldn = ldn;
  a.H = H;
  a.mbf = (float)(-0.5 * (double)bfactor / n / n);
  a.inv_size = (float)(1.0 / ((double)(n / 2 + 1) * n));
  a.P = P;
  a.Q = Q;
  a.twO = two;
  a.box = pbx;
  a.ystart = ystart;
  a.G = G;
  if (mc::launch_pair_cols(a, st) != cudaSuccess) return fail(MC_E_CUDA, "column stage launch failed");
  mc::PairRowsArgs r{};
  r.G = G;
  r.npairs = 1;
  r.H = H;
  r.box = pbx;
  r.cs = cs;
  r.boxes = d_window;
  if (mc::launch_pair_rows(r, st) != cudaSuccess) return fail(MC_E_CUDA, "row stage launch failed");
  return MC_OK;
}

}  // extern "C"
