// Hand-written sm_100a kernels of the drift-correction path.
//
//   k_fwd_rows    decode + dark/gain + crop + row R2C, transposed store    (DFAlign.cu:710-806)
//   k_rows_fft    batched row FFTs: forward column pass with Fourier-crop binning
//                 (cufunc.cu:162-176, 223-227) and the inverse passes
//   k_pair_cols   cross-power x B-factor + pruned inverse FFT along ky     (cufunc.cu:343-370)
//   k_pair_rows   pruned C2R along kx onto the pbx window                  (cufunc.cu:229-233, 404-407)
//   k_peak        integer peak + x32 Fourier-upsampled sub-pixel peak     (cufunc.cu:396-497)
//   k_shift_sum   phase-shift-and-accumulate (+ inverse column FFT)       (cufunc.cu:372-393)
//   k_c2r_rows    final C2R rows x 1/n^2                                   (DFAlign.cu:1287-1292)
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "kernels.cuh"
#include "codelets_gen.cuh"

namespace mc {

// Raise-only, thread-safe opt-in to large dynamic shared memory.  The
// attribute is per function and per device; two host threads that launch
// the same kernel with different sizes must never lower it under each other.
cudaError_t allow_smem(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = done[{dev, func}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float load_pixel(const void* frame, int mode, long long idx) {
  switch (mode) {
    case 0: return (float)((const int8_t*)frame)[idx];
    case 1: return (float)((const int16_t*)frame)[idx];
    case 6: return (float)((const uint16_t*)frame)[idx];
    default: return ((const float*)frame)[idx];
  }
}

// exp(+/-2 pi i m / len) tables live in shared memory for the whole kernel.
__device__ __forceinline__ void copy_table(float2* dst, const float2* __restrict__ src, int cnt) {
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) dst[i] = src[i];
}

}  // namespace

// Frame read by a forward launch (direct pointer, or the run's base from the
// device-side slot plus this frame's offset).
__device__ __forceinline__ const void* fwd_frame(const FwdRowsArgs& a) {
  return a.frames_slot ? static_cast<const void*>(static_cast<const char*>(*a.frames_slot) + a.frame_offset)
                       : a.frame;
}

// =========================================================== forward rows ==
__global__ void __launch_bounds__(kThreads) k_fwd_rows(FwdRowsArgs a) {
  const void* frame = fwd_frame(a);
  extern __shared__ float2 sm[];
  const int nu = a.nu;
  float2* b0 = sm;
  float2* b1 = sm + nu;
  float2* tw = sm + 2 * nu;
  copy_table(tw, a.tw, nu);
  const int tid = threadIdx.x, nth = blockDim.x;
  // rows handled by this CTA
  int y0, y1;
  if (a.two_outputs) {
    y0 = blockIdx.x;
    y1 = y0;
  } else {
    y0 = 2 * blockIdx.x;
    y1 = y0 + 1;
  }
  const bool hasd = a.dark != nullptr, hasn = a.norm != nullptr;
  const long long r0 = (long long)(a.offy + y0) * a.nx + a.offx;
  const long long r1 = (long long)(a.offy + y1) * a.nx + a.offx;
  for (int x = tid; x < nu; x += nth) {
    float re, im;
    if (a.two_outputs) {
      const long long i0 = r0 + x;
      const float raw = load_pixel(frame, a.mode, i0);
      const float d1 = hasd ? a.dark[i0] : 0.f;
      const float d2 = hasd ? (a.dark2 ? a.dark2[i0] : 0.f) : 0.f;
      const float g1 = hasn ? a.norm[i0] : 1.f;
      const float g2 = hasn ? (a.norm2 ? a.norm2[i0] : 1.f) : 1.f;
      re = (raw - d1) * g1;  // hbuf   (DFAlign.cu:725)
      im = (raw - d2) * g2;  // hbuf2  (DFAlign.cu:724)
    } else {
      re = load_pixel(frame, a.mode, r0 + x);
      im = load_pixel(frame, a.mode, r1 + x);
      if (hasd || hasn) {  // identical references: one spectrum per frame
        const long long i0 = r0 + x, i1 = r1 + x;
        re = (re - (hasd ? a.dark[i0] : 0.f)) * (hasn ? a.norm[i0] : 1.f);
        im = (im - (hasd ? a.dark[i1] : 0.f)) * (hasn ? a.norm[i1] : 1.f);
      }
    }
    b0[x] = make_float2(re, im);
  }
  __syncthreads();
  float2* Z = fft_run<false, false>(b0, b1, a.plan, 1, nu, tw, tid, nth);
  // split the two real transforms: X = (Z(k) + conj Z(-k))/2, Y = -i (Z(k) - conj Z(-k))/2
  for (int k = tid; k < a.hk; k += nth) {
    const float2 z = Z[k];
    const float2 zc = Z[k == 0 ? 0 : nu - k];
    const float2 X = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    const float2 Y = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
    if (a.two_outputs) {
      a.outA[(long long)k * a.ldt + y0] = X;
      a.outB[(long long)k * a.ldt + y0] = Y;
    } else {
      float4* dst = reinterpret_cast<float4*>(a.outA + (long long)k * a.ldt + y0);
      *dst = make_float4(X.x, X.y, Y.x, Y.y);
    }
  }
}

size_t fwd_rows_smem(int nu) { return (size_t)3 * nu * sizeof(float2); }

bool two_level_split(int n, int& n1, int& n2);
cudaError_t launch_fwd_rows2l(const FwdRowsArgs& a, cudaStream_t st);
cudaError_t launch_rows_fft2l(const RowsFftArgs& a, bool inverse, cudaStream_t st);

cudaError_t launch_fwd_rows_dif(const FwdRowsArgs& a, cudaStream_t st);
cudaError_t launch_rows_fft_dif(const RowsFftArgs& a, cudaStream_t st);
bool dif_supported(int n);

cudaError_t launch_fwd_rows(const FwdRowsArgs& a, cudaStream_t st) {
  int n1, n2;
  if (two_level_split(a.nu, n1, n2)) return launch_fwd_rows2l(a, st);
  const bool raw = !a.two_outputs && !a.dark && !a.dark2 && !a.norm && !a.norm2;
  if (raw && dif_supported(a.nu)) return launch_fwd_rows_dif(a, st);
  const size_t smem = fwd_rows_smem(a.nu);
  cudaError_t e = allow_smem((const void*)k_fwd_rows, smem);
  if (e != cudaSuccess) return e;
  const int grid = a.two_outputs ? a.nu : a.nu / 2;
  k_fwd_rows<<<grid, kThreads, smem, st>>>(a);
  return cudaGetLastError();
}

// ========================================================= row transforms ==
template <bool INV>
__global__ void __launch_bounds__(kThreads) k_rows_fft(RowsFftArgs a, int rows_per_cta) {
  extern __shared__ float2 sm[];
  const int n = a.plan.n;
  const int B = rows_per_cta;
  float2* b0 = sm;
  float2* b1 = sm + (size_t)B * n;
  float2* tw = sm + (size_t)2 * B * n;
  copy_table(tw, a.tw, n);
  const int tid = threadIdx.x, nth = blockDim.x;
  const int row0 = blockIdx.x * B;
  const int nb = min(B, a.nrows - row0);
  for (int t = tid; t < B * n; t += nth) {
    const int b = t / n, i = t - b * n;
    b0[t] = (b < nb) ? a.in[(long long)(row0 + b) * a.ld_in + i] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* X = fft_run<INV, false>(b0, b1, a.plan, B, n, tw, tid, nth);
  const int shift = n - a.n_out;
  for (int t = tid; t < nb * a.n_out; t += nth) {
    const int b = t / a.n_out, i = t - b * a.n_out;
    const int src = (i < a.keep_lo) ? i : i + shift;
    const float2 v = X[b * n + src];
    a.out[(long long)(row0 + b) * a.ld_out + i] = make_float2(v.x * a.scale, v.y * a.scale);
  }
}

size_t rows_fft_smem(int n, int rows_per_cta) {
  return (size_t)(2 * rows_per_cta + 1) * n * sizeof(float2);
}

cudaError_t launch_rows_fft(const RowsFftArgs& a, bool inverse, int rows_per_cta, cudaStream_t st) {
  int n1, n2;
  if (two_level_split(a.plan.n, n1, n2)) return launch_rows_fft2l(a, inverse, st);
  if (!inverse && dif_supported(a.plan.n)) return launch_rows_fft_dif(a, st);
  const size_t smem = rows_fft_smem(a.plan.n, rows_per_cta);
  const int grid = (a.nrows + rows_per_cta - 1) / rows_per_cta;
  cudaError_t e;
  if (inverse) {
    e = allow_smem((const void*)k_rows_fft<true>, smem);
    if (e != cudaSuccess) return e;
    k_rows_fft<true><<<grid, kThreads, smem, st>>>(a, rows_per_cta);
  } else {
    e = allow_smem((const void*)k_rows_fft<false>, smem);
    if (e != cudaSuccess) return e;
    k_rows_fft<false><<<grid, kThreads, smem, st>>>(a, rows_per_cta);
  }
  return cudaGetLastError();
}

// ================================================== two-level transforms ==
// Length N = N1*N2 with n = n1 + N1*n2 and k = k2 + N2*k1:
//   Y[n1][k2]      = W_N^(n1 k2) * sum_n2 x[n1 + N1 n2] W_N2^(n2 k2)   thread n1: N2-point codelet
//   X[k2 + N2 k1]  = sum_n1 Y[n1][k2] W_N1^(n1 k1)                    thread k2: N1-point codelet
// so a whole transform costs one shared-memory exchange.  N1 = 53 uses the
// generated radix-53 butterfly.  One CTA (a team of `T2L` threads) per
// transform; W_N comes from the global twiddle table through the L1.
template <int N1, bool INV>
__device__ __forceinline__ void fft_n1(float2* v) {
  if constexpr (N1 == 53) dft_r53<INV>(v);
  else fft_reg<N1, INV>(v);
}

// Resident CTAs per SM the two-level transforms are compiled for (register cap).
// MC_FWD_PAIRED / MC_COL_PAIRED: two radix-53 output pairs per loop iteration
// in the forward row / column transforms.
#ifndef MC_FWD_PAIRED
#define MC_FWD_PAIRED false
#endif
#ifndef MC_COL_PAIRED
#define MC_COL_PAIRED false
#endif
#ifndef MC_TL_MIN_BLOCKS
#define MC_TL_MIN_BLOCKS 4
#endif

template <int N1, int N2>
struct TwoLevel {
  static constexpr int N = N1 * N2;
  static constexpr int T = ((N1 > N2 ? N1 : N2) + 31) / 32 * 32;

  // step A + exchange + step B; load(i) gives x[i], store(k, X[k]) takes the
  // result; tw[TWS * j] = exp(-2 pi i j / N).  For N1 = 53 only the outputs
  // with k1 or N1 - k1 <= kmax are formed (pruned transforms).  T >= N2, so each thread owns at most one k2 in step B; with
  // SYNC_STORE a barrier follows every thread's step-B reads of ysm, which
  // lets store() write back into ysm.
  template <bool INV, bool SYNC_STORE, bool PAIRED = false, int TWS = 1, class Load, class Store>
  __device__ static void run(float2* ysm, const float2* __restrict__ tw, Load&& load, Store&& store,
                             int kmax = (N1 - 1) / 2) {
    static_assert(T >= N2, "one k2 per thread");
    const int lt = threadIdx.x;
    if (lt < N1) {
      float2 x[N2];
#pragma unroll
      for (int n2 = 0; n2 < N2; n2++) x[n2] = load(lt + N1 * n2);
      fft_reg<N2, INV>(x);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) {
        float2 w = __ldg(tw + TWS * lt * k2);
        if (INV) w.y = -w.y;
        ysm[k2 * N1 + lt] = k2 ? cmul(x[k2], w) : x[k2];
      }
    }
    __syncthreads();
    const bool act = lt < N2;
    float2 v[N1];
    if (act) {
#pragma unroll
      for (int n1 = 0; n1 < N1; n1++) v[n1] = ysm[lt * N1 + n1];
    }
    if (SYNC_STORE) __syncthreads();
    if constexpr (N1 == 53) {
      // compact radix-53 DFT: small code, outputs stored as they are formed
      if (act) dft_r53_compact<INV, PAIRED>(v, [&](int k1, float2 x) { store(lt + N2 * k1, x); }, kmax);
    } else {
      if (act) fft_n1<N1, INV>(v);
      if (act) {
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) store(lt + N2 * k1, v[k1]);
      }
    }
  }
};

// Batched rows: out_row[i] = scale * X[i < keep_lo ? i : i + (n - n_out)].
template <int N1, int N2, bool INV>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS) k_rows_fft2l(RowsFftArgs a) {
  using TL = TwoLevel<N1, N2>;
  __shared__ float2 ysm[TL::N];
  const long long row = blockIdx.x;
  const float2* in = a.in + row * a.ld_in;
  float2* out = a.out + row * a.ld_out;
  const int shift = TL::N - a.n_out, keep = a.keep_lo;
  const float sc = a.scale;
  TL::template run<INV, false, MC_COL_PAIRED>(ysm, a.tw, [&](int i) { return __ldg(in + i); },
                        [&](int k, float2 v) {
                          int o;
                          if (k < keep) o = k;
                          else if (k >= keep + shift) o = k - shift;
                          else return;
                          out[o] = make_float2(v.x * sc, v.y * sc);
                        });
}

// Forward rows: two image rows (or the two reference sets of one row) packed
// as one complex transform, then split into the two real half spectra.
// Stage the two packed input rows of k_fwd_rows2l in shared memory: every
// thread of the CTA issues independent typed loads of the raw pixels.
template <typename Px>
__device__ __forceinline__ void stage_rows(float2* xin, const FwdRowsArgs& a, long long r0, long long r1, int n,
                                           int nth) {
  const Px* f = reinterpret_cast<const Px*>(fwd_frame(a));
  const bool hasd = a.dark != nullptr, hasn = a.norm != nullptr;
  if (a.two_outputs) {
#pragma unroll 4
    for (int x = threadIdx.x; x < n; x += nth) {
      const long long i0 = r0 + x;
      const float raw = (float)f[i0];
      const float d1 = hasd ? a.dark[i0] : 0.f;
      const float d2 = hasd ? (a.dark2 ? a.dark2[i0] : 0.f) : 0.f;
      const float g1 = hasn ? a.norm[i0] : 1.f;
      const float g2 = hasn ? (a.norm2 ? a.norm2[i0] : 1.f) : 1.f;
      xin[x] = make_float2((raw - d1) * g1, (raw - d2) * g2);  // hbuf, hbuf2 (DFAlign.cu:724-725)
    }
  } else if (hasd || hasn) {
#pragma unroll 4
    for (int x = threadIdx.x; x < n; x += nth) {
      const long long i0 = r0 + x, i1 = r1 + x;
      const float re = ((float)f[i0] - (hasd ? a.dark[i0] : 0.f)) * (hasn ? a.norm[i0] : 1.f);
      const float im = ((float)f[i1] - (hasd ? a.dark[i1] : 0.f)) * (hasn ? a.norm[i1] : 1.f);
      xin[x] = make_float2(re, im);
    }
  } else {
#pragma unroll 8
    for (int x = threadIdx.x; x < n; x += nth) xin[x] = make_float2((float)f[r0 + x], (float)f[r1 + x]);
  }
}

// Raw pixels of one crop row into shared memory with aligned 16-byte loads:
// the bytes of [src, src + n) land at dst[d + i] with d = src mod 16, so
// every interior 16-byte chunk keeps its alignment in shared memory; the
// unaligned head and tail go pixel by pixel.  Every load stays inside the row.
template <typename Px>
__device__ __forceinline__ void stage_raw_row(unsigned char* dst, const Px* src, int n, int tid, int nth) {
  const uintptr_t s = reinterpret_cast<uintptr_t>(src);
  const uintptr_t e = s + (uintptr_t)n * sizeof(Px);
  const uintptr_t a0 = s & ~(uintptr_t)15;
  uintptr_t as = (s + 15) & ~(uintptr_t)15;
  uintptr_t ae = e & ~(uintptr_t)15;
  if (as > ae) as = ae = e;  // row shorter than one aligned chunk: all pixel by pixel
  const int head = (int)((as - s) / sizeof(Px)), tail0 = (int)((ae - s) / sizeof(Px));
  Px* dpx = reinterpret_cast<Px*>(dst + (s - a0));
  for (int i = tid; i < head; i += nth) dpx[i] = src[i];
  for (int i = tail0 + tid; i < n; i += nth) dpx[i] = src[i];
  const int chunks = (int)((ae - as) / 16);
  const uint4* g = reinterpret_cast<const uint4*>(as);
  uint4* d4 = reinterpret_cast<uint4*>(dst + (as - a0));
  for (int c = tid; c < chunks; c += nth) d4[c] = __ldg(g + c);
}

// Shared bytes one staged row takes: n pixels + up to 15 bytes of alignment,
// rounded to 16.
template <typename Px>
constexpr int raw_row_bytes(int n) {
  return (n * (int)sizeof(Px) + 15 + 15) / 16 * 16;
}

// Forward rows without references: two rows staged as raw pixels (a quarter
// of the float staging for 8-bit frames), decoded in the step-A loads; the
// spectrum Z is written back into the exchange buffer after the barrier that
// follows the step-B reads.
template <int N1, int N2, typename Px>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS) k_fwd_rows2l_raw(FwdRowsArgs a) {
  using TL = TwoLevel<N1, N2>;
  constexpr int N = TL::N;
  constexpr int RB = raw_row_bytes<Px>(N);
  extern __shared__ float2 dynraw[];
  float2* ysm = dynraw;
  unsigned char* raw0 = reinterpret_cast<unsigned char*>(dynraw + N);
  unsigned char* raw1 = raw0 + RB;
  const int y0 = 2 * blockIdx.x, y1 = y0 + 1;
  const Px* f = reinterpret_cast<const Px*>(fwd_frame(a));
  const Px* row0 = f + (long long)(a.offy + y0) * a.nx + a.offx;
  const Px* row1 = f + (long long)(a.offy + y1) * a.nx + a.offx;
  stage_raw_row<Px>(raw0, row0, N, threadIdx.x, TL::T);
  stage_raw_row<Px>(raw1, row1, N, threadIdx.x, TL::T);
  __syncthreads();
  const Px* p0 = reinterpret_cast<const Px*>(raw0 + (reinterpret_cast<uintptr_t>(row0) & 15));
  const Px* p1 = reinterpret_cast<const Px*>(raw1 + (reinterpret_cast<uintptr_t>(row1) & 15));
  TL::template run<false, true, MC_FWD_PAIRED>(
      ysm, a.tw, [&](int x) { return make_float2((float)p0[x], (float)p1[x]); },
      [&](int k, float2 v) { ysm[k] = v; });
  __syncthreads();
  for (int k = threadIdx.x; k < a.hk; k += TL::T) {
    const float2 z = ysm[k];
    const float2 zc = ysm[k == 0 ? 0 : N - k];
    const float2 X = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    const float2 Y = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
    *reinterpret_cast<float4*>(a.outA + (long long)k * a.ldt + y0) = make_float4(X.x, X.y, Y.x, Y.y);
  }
}

template <int N1, int N2>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS) k_fwd_rows2l(FwdRowsArgs a) {
  using TL = TwoLevel<N1, N2>;
  constexpr int N = TL::N;
  extern __shared__ float2 dyn2l[];
  float2* xin = dyn2l;      // packed input rows, later the spectrum Z
  float2* ysm = dyn2l + N;  // exchange buffer
  int y0, y1;
  if (a.two_outputs) {
    y0 = blockIdx.x;
    y1 = y0;
  } else {
    y0 = 2 * blockIdx.x;
    y1 = y0 + 1;
  }
  const long long r0 = (long long)(a.offy + y0) * a.nx + a.offx;
  const long long r1 = (long long)(a.offy + y1) * a.nx + a.offx;
  switch (a.mode) {
    case 0: stage_rows<int8_t>(xin, a, r0, r1, N, TL::T); break;
    case 1: stage_rows<int16_t>(xin, a, r0, r1, N, TL::T); break;
    case 6: stage_rows<uint16_t>(xin, a, r0, r1, N, TL::T); break;
    default: stage_rows<float>(xin, a, r0, r1, N, TL::T); break;
  }
  __syncthreads();
  // step B writes Z into xin: every step-A read of xin precedes the barrier
  // between the steps, and step B reads only ysm
  float2* zsm = xin;
  TL::template run<false, false>(
      ysm, a.tw, [&](int x) { return xin[x]; }, [&](int k, float2 v) { zsm[k] = v; });
  __syncthreads();
  for (int k = threadIdx.x; k < a.hk; k += TL::T) {
    const float2 z = zsm[k];
    const float2 zc = zsm[k == 0 ? 0 : N - k];
    const float2 X = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    const float2 Y = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
    if (a.two_outputs) {
      a.outA[(long long)k * a.ldt + y0] = X;
      a.outB[(long long)k * a.ldt + y0] = Y;
    } else {
      *reinterpret_cast<float4*>(a.outA + (long long)k * a.ldt + y0) = make_float4(X.x, X.y, Y.x, Y.y);
    }
  }
}

// ---------------------------------------------------------------------------
// Lengths L = 2N with a two-level N (7420 = 2 x 3710 at -bin 2): one radix-2
// decimation-in-frequency step folded into the step-A loads,
//   A[m] = FFT_N(z_n + z_{n+N})[m] = Z[2m],
//   B[m] = FFT_N((z_n - z_{n+N}) W_L^n)[m] = Z[2m+1],
// then the two N-point two-level transforms, whose outputs go straight to
// the kept indices.  tw is the L-entry table exp(-2 pi i j / L).

// Output pairs (k1, N1 - k1) of the N1-point step a radix-2 split transform
// needs when only its outputs below `lo` (2m < lo) and their mirror images
// (2m > L - lo) are kept: m = k2 + N2*k1 < lo/2 needs k1 <= (lo/2 - 1)/N2,
// one more pair for the boundary row; all pairs when that reaches (N1-1)/2.
template <int N1, int N2>
__device__ __forceinline__ int dif_kmax(int lo) {
  const int k = (lo / 2) / N2 + 1;
  return k < (N1 - 1) / 2 ? k : (N1 - 1) / 2;
}

// Forward rows of length L without references: two rows staged as raw
// pixels; only the Z indices the half-spectrum split needs are kept in
// shared memory (Z[0, hk) and Z(L - hk, L)).
template <int N1, int N2, typename Px>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS) k_fwd_rows_dif(FwdRowsArgs a) {
  using TL = TwoLevel<N1, N2>;
  constexpr int N = TL::N, L = 2 * N;
  constexpr int RB = raw_row_bytes<Px>(L);
  extern __shared__ float2 dyndif[];
  const int hk = a.hk;
  float2* ysm = dyndif;
  float2* zlo = dyndif + N;   // Z[0 .. hk-1]
  float2* zhi = zlo + hk;     // Z[L-hk+1 .. L-1]
  unsigned char* raw0 = reinterpret_cast<unsigned char*>(zhi + hk);
  unsigned char* raw1 = raw0 + RB;
  const int y0 = 2 * blockIdx.x, y1 = y0 + 1;
  const Px* f = reinterpret_cast<const Px*>(fwd_frame(a));
  const Px* row0 = f + (long long)(a.offy + y0) * a.nx + a.offx;
  const Px* row1 = f + (long long)(a.offy + y1) * a.nx + a.offx;
  stage_raw_row<Px>(raw0, row0, L, threadIdx.x, TL::T);
  stage_raw_row<Px>(raw1, row1, L, threadIdx.x, TL::T);
  __syncthreads();
  const Px* p0 = reinterpret_cast<const Px*>(raw0 + (reinterpret_cast<uintptr_t>(row0) & 15));
  const Px* p1 = reinterpret_cast<const Px*>(raw1 + (reinterpret_cast<uintptr_t>(row1) & 15));
  const float2* tw = a.tw;
  auto keep = [&](int idx, float2 v) {
    if (idx < hk) zlo[idx] = v;
    else if (idx > L - hk) zhi[idx - (L - hk + 1)] = v;
  };
  // wanted A/B outputs: m < hk/2 or m > N - hk/2, i.e. m = k2 + N2*k1 with
  // k1 or N1 - 1 - k1 at most (hk/2)/N2
  const int kmax = dif_kmax<N1, N2>(hk);
  TL::template run<false, false, false, 2>(
      ysm, tw,
      [&](int n) {
        return make_float2((float)p0[n] + (float)p0[n + N], (float)p1[n] + (float)p1[n + N]);
      },
      [&](int m, float2 v) { keep(2 * m, v); }, kmax);
  __syncthreads();
  TL::template run<false, false, false, 2>(
      ysm, tw,
      [&](int n) {
        const float2 d = make_float2((float)p0[n] - (float)p0[n + N], (float)p1[n] - (float)p1[n + N]);
        return cmul(d, __ldg(tw + n));
      },
      [&](int m, float2 v) { keep(2 * m + 1, v); }, kmax);
  __syncthreads();
  for (int k = threadIdx.x; k < hk; k += TL::T) {
    const float2 z = zlo[k];
    const float2 zc = k == 0 ? zlo[0] : zhi[hk - 1 - k];
    const float2 X = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    const float2 Y = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
    *reinterpret_cast<float4*>(a.outA + (long long)k * a.ldt + y0) = make_float4(X.x, X.y, Y.x, Y.y);
  }
}

// Forward columns of length L: out_row[i] = scale * X[i < keep_lo ? i : i + (L - n_out)].
template <int N1, int N2>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS) k_rows_fft_dif(RowsFftArgs a) {
  using TL = TwoLevel<N1, N2>;
  constexpr int N = TL::N, L = 2 * N;
  __shared__ float2 ysm[N];
  const long long row = blockIdx.x;
  const float2* in = a.in + row * a.ld_in;
  float2* out = a.out + row * a.ld_out;
  const int shift = L - a.n_out, keep = a.keep_lo;
  const float sc = a.scale;
  const float2* tw = a.tw;
  auto put = [&](int i, float2 v) {
    int o;
    if (i < keep) o = i;
    else if (i >= keep + shift) o = i - shift;
    else return;
    out[o] = make_float2(v.x * sc, v.y * sc);
  };
  // wanted outputs i < keep or i >= keep + shift: with no crop all of them
  const int kmax = shift == 0 ? (N1 - 1) / 2 : dif_kmax<N1, N2>(keep + 1);
  TL::template run<false, false, false, 2>(
      ysm, tw, [&](int n) { return cadd(__ldg(in + n), __ldg(in + n + N)); },
      [&](int m, float2 v) { put(2 * m, v); }, kmax);
  __syncthreads();
  TL::template run<false, false, false, 2>(
      ysm, tw,
      [&](int n) {
        const float2 x0 = __ldg(in + n), x1 = __ldg(in + n + N);
        return cmul(make_float2(x0.x - x1.x, x0.y - x1.y), __ldg(tw + n));
      },
      [&](int m, float2 v) { put(2 * m + 1, v); }, kmax);
}

// Two-level splits compiled in (N1, N2).
#define MC_TWO_LEVEL_LIST(X) X(53, 70) X(64, 64) X(32, 64) X(32, 32) X(16, 16) X(16, 32)

bool two_level_split(int n, int& n1, int& n2) {
#define MC_TL_MATCH(A, B)      \
  if (n == (A) * (B)) {        \
    n1 = (A);                  \
    n2 = (B);                  \
    return true;               \
  }
  MC_TWO_LEVEL_LIST(MC_TL_MATCH)
#undef MC_TL_MATCH
  return false;
}

cudaError_t launch_rows_fft2l(const RowsFftArgs& a, bool inverse, cudaStream_t st) {
  int n1 = 0, n2 = 0;
  if (!two_level_split(a.plan.n, n1, n2)) return cudaErrorInvalidValue;
#define MC_TL_LAUNCH(A, B)                                                                   \
  if (n1 == (A) && n2 == (B)) {                                                              \
    if (inverse) k_rows_fft2l<A, B, true><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a);         \
    else k_rows_fft2l<A, B, false><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a);                \
    return cudaGetLastError();                                                               \
  }
  MC_TWO_LEVEL_LIST(MC_TL_LAUNCH)
#undef MC_TL_LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_rows2l(const FwdRowsArgs& a, cudaStream_t st) {
  int n1 = 0, n2 = 0;
  if (!two_level_split(a.nu, n1, n2)) return cudaErrorInvalidValue;
  const int grid = a.two_outputs ? a.nu : a.nu / 2;
  const bool raw = !a.two_outputs && !a.dark && !a.dark2 && !a.norm && !a.norm2;
#define MC_TL_RAW(A, B, PX)                                                                          \
  {                                                                                                  \
    const size_t smem = (size_t)(A) * (B) * sizeof(float2) + 2 * (size_t)raw_row_bytes<PX>((A) * (B)); \
    cudaError_t e = allow_smem((const void*)k_fwd_rows2l_raw<A, B, PX>, smem);                       \
    if (e != cudaSuccess) return e;                                                                  \
    k_fwd_rows2l_raw<A, B, PX><<<grid, TwoLevel<A, B>::T, smem, st>>>(a);                            \
    return cudaGetLastError();                                                                       \
  }
#define MC_TL_LAUNCH(A, B)                                                                           \
  if (n1 == (A) && n2 == (B)) {                                                                      \
    if (raw) {                                                                                       \
      switch (a.mode) {                                                                              \
        case 0: MC_TL_RAW(A, B, int8_t)                                                              \
        case 1: MC_TL_RAW(A, B, int16_t)                                                             \
        case 6: MC_TL_RAW(A, B, uint16_t)                                                            \
        default: MC_TL_RAW(A, B, float)                                                              \
      }                                                                                              \
    }                                                                                                \
    const size_t smem = (size_t)2 * (A) * (B) * sizeof(float2);                                      \
    cudaError_t e = allow_smem((const void*)k_fwd_rows2l<A, B>, smem);                               \
    if (e != cudaSuccess) return e;                                                                  \
    k_fwd_rows2l<A, B><<<grid, TwoLevel<A, B>::T, smem, st>>>(a);                                    \
    return cudaGetLastError();                                                                       \
  }
  MC_TWO_LEVEL_LIST(MC_TL_LAUNCH)
#undef MC_TL_LAUNCH
#undef MC_TL_RAW
  return cudaErrorInvalidValue;
}

bool dif_supported(int n) {
  int n1, n2;
  return n % 2 == 0 && two_level_split(n / 2, n1, n2);
}

cudaError_t launch_fwd_rows_dif(const FwdRowsArgs& a, cudaStream_t st) {
  int n1 = 0, n2 = 0;
  if (a.nu % 2 || !two_level_split(a.nu / 2, n1, n2)) return cudaErrorInvalidValue;
  const int grid = a.nu / 2;
#define MC_DIF_RAW(A, B, PX)                                                                          \
  {                                                                                                   \
    const size_t smem = ((size_t)(A) * (B) + 2 * (size_t)a.hk) * sizeof(float2) +                     \
                        2 * (size_t)raw_row_bytes<PX>(2 * (A) * (B));                                 \
    cudaError_t e = allow_smem((const void*)k_fwd_rows_dif<A, B, PX>, smem);                          \
    if (e != cudaSuccess) return e;                                                                   \
    k_fwd_rows_dif<A, B, PX><<<grid, TwoLevel<A, B>::T, smem, st>>>(a);                               \
    return cudaGetLastError();                                                                        \
  }
#define MC_DIF_LAUNCH(A, B)                                                                           \
  if (n1 == (A) && n2 == (B)) {                                                                       \
    switch (a.mode) {                                                                                 \
      case 0: MC_DIF_RAW(A, B, int8_t)                                                                \
      case 1: MC_DIF_RAW(A, B, int16_t)                                                               \
      case 6: MC_DIF_RAW(A, B, uint16_t)                                                              \
      default: MC_DIF_RAW(A, B, float)                                                                \
    }                                                                                                 \
  }
  MC_TWO_LEVEL_LIST(MC_DIF_LAUNCH)
#undef MC_DIF_LAUNCH
#undef MC_DIF_RAW
  return cudaErrorInvalidValue;
}

cudaError_t launch_rows_fft_dif(const RowsFftArgs& a, cudaStream_t st) {
  int n1 = 0, n2 = 0;
  if (a.plan.n % 2 || !two_level_split(a.plan.n / 2, n1, n2)) return cudaErrorInvalidValue;
#define MC_DIF_LAUNCH(A, B)                                                        \
  if (n1 == (A) && n2 == (B)) {                                                    \
    k_rows_fft_dif<A, B><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a);                \
    return cudaGetLastError();                                                     \
  }
  MC_TWO_LEVEL_LIST(MC_DIF_LAUNCH)
#undef MC_DIF_LAUNCH
  return cudaErrorInvalidValue;
}

// ============================================================ pair columns ==
size_t pair_cols_smem(int n, int P, int Q, int box) {
  return (size_t)2 * n * sizeof(float2)       // ping-pong
         + (size_t)n * sizeof(float)          // B-factor column
         + (size_t)Q * sizeof(float2)         // inner twiddles
         + (size_t)P * box * sizeof(float2);  // outer twiddles
}

__global__ void __launch_bounds__(kThreads) k_pair_cols(PairColsArgs a) {
  extern __shared__ float2 sm[];
  const int n = a.n, P = a.P, Q = a.Q, box = a.box;
  float2* x0 = sm;
  float2* x1 = sm + n;
  float* wcol = reinterpret_cast<float*>(sm + 2 * n);
  float2* twQ = reinterpret_cast<float2*>(wcol + n + (n & 1));  // keep 8-byte alignment
  float2* twO = twQ + Q;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int kx = blockIdx.y;
  copy_table(twQ, a.twQ, Q);
  copy_table(twO, a.twO, P * box);
  const int half = n / 2;
  for (int ky = tid; ky < n; ky += nth) {
    const int y = ky < half ? ky : ky - n;
    const float r2 = (float)(kx * kx + y * y);
    wcol[ky] = expf(a.mbf * r2) * a.inv_size;
  }
  __syncthreads();
  const int p0 = blockIdx.x * a.pairs_per_cta;
  const int p1 = min(p0 + a.pairs_per_cta, a.npairs);
  const int nout = box * 2;  // two threads per output (k1 halves)
  const int khalf = (P + 1) / 2;
  for (int p = p0; p < p1; p++) {
    const int2 pr = a.pairs[p];
    const float2* ca = a.specA + (long long)pr.x * a.strideA + (long long)kx * a.ldn;
    const float2* cb = a.specB + (long long)pr.y * a.strideB + (long long)kx * a.ldn;
    for (int ky = tid; ky < n; ky += nth) {
      const float2 u = ca[ky], v = cb[ky];
      x0[ky] = cscale(cmulc(u, v), wcol[ky]);
    }
    __syncthreads();
    const float2* Y = fft_run<true, true>(x0, x1, a.qplan, P, 0, twQ, tid, nth);
    for (int base = 0; base < nout; base += nth) {
      const int o = base + tid;
      const bool ok = o < nout;
      const int m = o >> 1, h = o & 1;
      float2 acc = make_float2(0.f, 0.f);
      if (ok) {
        const int r = (a.ystart + m) % Q;
        const int k0 = h ? khalf : 0, k1 = h ? P : khalf;
        const float2* yr = Y + (long long)P * r;
        for (int k = k0; k < k1; k++) {
          const float2 t = twO[k * box + m];
          const float2 yv = yr[k];
          acc.x = fmaf(t.x, yv.x, fmaf(-t.y, yv.y, acc.x));
          acc.y = fmaf(t.x, yv.y, fmaf(t.y, yv.x, acc.y));
        }
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
      if (ok && h == 0) a.G[((long long)p * a.H + kx) * box + m] = acc;
    }
    __syncthreads();
  }
}

// Register-codelet variant of the column stage (P <= 128, Q a codelet length).
// A CTA of 128 threads owns one column kx; it is split into teams of `team`
// threads (team = P rounded up to a warp multiple) and each team takes whole
// pairs.  Thread k1 < P of a team gathers its stride-P subsequence
// c(k1 + P*k2), k2 < Q, straight from the two spectra (coalesced over k1),
// runs the Q-point inverse FFT in registers, and parks the result in shared
// memory; the team then forms the pbx output rows as P-term sums.
constexpr int kRegThreads = 128;

__device__ __forceinline__ void team_barrier(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

size_t pair_cols_reg_smem(int n, int team) {
  const int teams = kRegThreads / team;
  return (size_t)((n + 1) / 2) * sizeof(float2) + (size_t)teams * n * sizeof(float2);
}

// Resident 128-thread CTAs per SM the one-thread-per-subsequence kernel is
// compiled for: four (128 registers) up to Q = 40, three (168) up to 56, two
// (255) above.
constexpr int pair_reg_min_blocks(int Q) { return Q <= 40 ? 4 : (Q <= 56 ? 3 : 2); }

template <int Q>
__global__ void __launch_bounds__(kRegThreads, pair_reg_min_blocks(Q)) k_pair_cols_reg(PairColsArgs a, int team) {
  extern __shared__ float2 sm[];
  const int n = a.n, P = a.P, box = a.box;
  float* wcol = reinterpret_cast<float*>(sm);
  const int teams = kRegThreads / team;
  const int tid = threadIdx.x;
  const int tm = tid / team, lt = tid - tm * team;
  float2* Y = sm + (n + 1) / 2 + (size_t)tm * n;
  const int kx = blockIdx.y;
  const int half = n / 2;
  for (int ky = tid; ky < n; ky += kRegThreads) {
    const int y = ky < half ? ky : ky - n;
    wcol[ky] = expf(a.mbf * (float)(kx * kx + y * y)) * a.inv_size;
  }
  __syncthreads();
  const int p0 = blockIdx.x * a.pairs_per_cta;
  const int p1 = min(p0 + a.pairs_per_cta, a.npairs);
  const int khalf = (P + 1) / 2;
  for (int p = p0 + tm; p < p1; p += teams) {
    const int2 pr = a.pairs[p];
    const float2* ca = a.specA + (long long)pr.x * a.strideA + (long long)kx * a.ldn;
    const float2* cb = a.specB + (long long)pr.y * a.strideB + (long long)kx * a.ldn;
    if (lt < P) {
      float2 x[Q];
#pragma unroll
      for (int k2 = 0; k2 < Q; k2++) {
        const int ky = lt + P * k2;
        x[k2] = cscale(cmulc(__ldg(ca + ky), __ldg(cb + ky)), wcol[ky]);
      }
      fft_reg<Q, true>(x);
#pragma unroll
      for (int r = 0; r < Q; r++) Y[lt + P * r] = x[r];
    }
    team_barrier(1 + tm, team);
    for (int base = 0; base < 2 * box; base += team) {
      const int o = base + lt;
      const bool ok = o < 2 * box;
      const int m = o >> 1, h = o & 1;
      float2 acc = make_float2(0.f, 0.f);
      if (ok) {
        const int r = (a.ystart + m) % Q;
        const int k0 = h ? khalf : 0, k1 = h ? P : khalf;
        const float2* yr = Y + P * r;
        const float2* tw = a.twO + m;
        for (int k = k0; k < k1; k++) {
          const float2 t = __ldg(tw + k * box);
          const float2 yv = yr[k];
          acc.x = fmaf(t.x, yv.x, fmaf(-t.y, yv.y, acc.x));
          acc.y = fmaf(t.x, yv.y, fmaf(t.y, yv.x, acc.y));
        }
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
      if (ok && h == 0) a.G[((long long)p * a.H + kx) * box + m] = acc;
    }
    team_barrier(1 + tm, team);
  }
}

// ---- grouped variant: one CTA per (A frame group, column kx) -------------
// The pairs of a batch come in groups that share their A spectrum (the
// reference's i-major order).  The CTA stages A(kx,:) x B-factor once in
// shared memory; each team double-buffers the B columns of its pairs with
// 16-byte cp.async copies, so the copy of pair p+1 overlaps the transform of
// pair p.  Thread k1 reads only positions k1 + P*k2 of the B buffer and
// writes Y back to the same positions, so Y lives in the consumed buffer.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

size_t pair_cols_grp_smem(int n, int teams) { return (size_t)(1 + 2 * teams) * n * sizeof(float2); }

template <int Q>
__global__ void __launch_bounds__(kRegThreads) k_pair_cols_grp(PairColsArgs a, const int2* __restrict__ groups,
                                                               int team) {
  extern __shared__ float2 smg[];
  const int n = a.n, P = a.P, box = a.box;
  const int teams = kRegThreads / team;
  const int tid = threadIdx.x;
  const int tm = tid / team, lt = tid - tm * team;
  float2* aw = smg;
  float2* buf0 = smg + n + (size_t)2 * tm * n;
  const int kx = blockIdx.y;
  const int2 g = groups[blockIdx.x];  // (first pair, count)
  const int half = n / 2;
  const int2 pr0 = a.pairs[g.x];
  const float2* ca = a.specA + (long long)pr0.x * a.strideA + (long long)kx * a.ldn;
  for (int ky = tid; ky < n; ky += kRegThreads) {
    const int y = ky < half ? ky : ky - n;
    const float w = expf(a.mbf * (float)(kx * kx + y * y)) * a.inv_size;
    aw[ky] = cscale(__ldg(ca + ky), w);
  }
  const int nchunk = n / 2;  // 16-byte chunks of a column (n is even)
  auto fetch = [&](int q, float2* dst) {
    const int2 pr = a.pairs[g.x + q];
    const float2* cb = a.specB + (long long)pr.y * a.strideB + (long long)kx * a.ldn;
    for (int c = lt; c < nchunk; c += team) cp_async16(dst + 2 * c, cb + 2 * c);
  };
  int cur = 0;
  if (tm < g.y) fetch(tm, buf0);
  cp_async_commit();
  __syncthreads();  // aw visible to every team
  const int khalf = (P + 1) / 2;
  for (int q = tm; q < g.y; q += teams) {
    float2* bc = buf0 + (size_t)cur * n;
    if (q + teams < g.y) fetch(q + teams, buf0 + (size_t)(cur ^ 1) * n);
    cp_async_commit();
    cp_async_wait<1>();
    team_barrier(1 + tm, team);
    if (lt < P) {
      float2 x[Q];
#pragma unroll
      for (int k2 = 0; k2 < Q; k2++) {
        const int ky = lt + P * k2;
        x[k2] = cmulc(aw[ky], bc[ky]);
      }
      fft_reg<Q, true>(x);
#pragma unroll
      for (int r = 0; r < Q; r++) bc[lt + P * r] = x[r];
    }
    team_barrier(1 + tm, team);
    const int p = g.x + q;
    for (int base = 0; base < 2 * box; base += team) {
      const int o = base + lt;
      const bool ok = o < 2 * box;
      const int m = o >> 1, h = o & 1;
      float2 acc = make_float2(0.f, 0.f);
      if (ok) {
        const int r = (a.ystart + m) % Q;
        const int k0 = h ? khalf : 0, k1 = h ? P : khalf;
        const float2* yr = bc + P * r;
        const float2* tw = a.twO + m;
        for (int k = k0; k < k1; k++) {
          const float2 t = __ldg(tw + k * box);
          const float2 yv = yr[k];
          acc.x = fmaf(t.x, yv.x, fmaf(-t.y, yv.y, acc.x));
          acc.y = fmaf(t.x, yv.y, fmaf(t.y, yv.x, acc.y));
        }
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
      if (ok && h == 0) a.G[((long long)p * a.H + kx) * box + m] = acc;
    }
    team_barrier(1 + tm, team);  // buffer `cur` may now be refilled
    cur ^= 1;
  }
  cp_async_wait<0>();
}

template <int Q>
cudaError_t launch_grp(const PairColsArgs& a, const int2* groups, int ngroups, int team, cudaStream_t st) {
  const size_t smem = pair_cols_grp_smem(a.n, kRegThreads / team);
  cudaError_t e = allow_smem((const void*)k_pair_cols_grp<Q>, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(ngroups, a.H);
  k_pair_cols_grp<Q><<<grid, kRegThreads, smem, st>>>(a, groups, team);
  return cudaGetLastError();
}

template <int I = 0>
cudaError_t dispatch_grp(const PairColsArgs& a, const int2* groups, int ngroups, int team, cudaStream_t st) {
  if constexpr (I < kNumCodelets) {
    constexpr int Q = kCodelets[I];
    if (a.Q == Q) return launch_grp<Q>(a, groups, ngroups, team, st);
    return dispatch_grp<I + 1>(a, groups, ngroups, team, st);
  } else {
    return cudaErrorInvalidValue;
  }
}

cudaError_t launch_pair_cols_grouped(const PairColsArgs& a, const int2* groups, int ngroups, int team,
                                     cudaStream_t st) {
  if (!pair_cols_reg_supported(a.P, a.Q) || (a.n & 1)) return cudaErrorInvalidValue;
  return dispatch_grp(a, groups, ngroups, team, st);
}

bool pair_cols_reg_supported(int P, int Q) {
  if (P < 1 || P > kRegThreads) return false;
  for (int q : kCodelets)
    if (q == Q) return true;
  return false;
}

template <int Q>
cudaError_t launch_reg(const PairColsArgs& a, int team, size_t smem, dim3 grid, cudaStream_t st) {
  cudaError_t e = allow_smem((const void*)k_pair_cols_reg<Q>, smem);
  if (e != cudaSuccess) return e;
  k_pair_cols_reg<Q><<<grid, kRegThreads, smem, st>>>(a, team);
  return cudaGetLastError();
}

template <int I = 0>
cudaError_t dispatch_reg(const PairColsArgs& a, int team, size_t smem, dim3 grid, cudaStream_t st) {
  if constexpr (I < kNumCodelets) {
    constexpr int Q = kCodelets[I];
    if (a.Q == Q) return launch_reg<Q>(a, team, smem, grid, st);
    return dispatch_reg<I + 1>(a, team, smem, grid, st);
  } else {
    return cudaErrorInvalidValue;
  }
}

cudaError_t launch_pair_cols(const PairColsArgs& a, cudaStream_t st) {
  dim3 grid((a.npairs + a.pairs_per_cta - 1) / a.pairs_per_cta, a.H);
  if (pair_cols_reg_supported(a.P, a.Q)) {
    const int team = a.P <= 32 ? 32 : (a.P <= 64 ? 64 : 128);
    return dispatch_reg(a, team, pair_cols_reg_smem(a.n, team), grid, st);
  }
  const size_t smem = pair_cols_smem(a.n, a.P, a.Q, a.box) + 16;
  cudaError_t e = allow_smem((const void*)k_pair_cols, smem);
  if (e != cudaSuccess) return e;
  k_pair_cols<<<grid, kThreads, smem, st>>>(a);
  return cudaGetLastError();
}

// =============================================================== pair rows ==
// 16x16 threads, each a 6x6 register tile of the 96x96 output block; kx in
// chunks of 32 staged through shared memory.
constexpr int kRowTile = 96;
constexpr int kRowK = 16;

__global__ void __launch_bounds__(kThreads) k_pair_rows(PairRowsArgs a) {
  __shared__ float2 gs[kRowK][kRowTile];
  __shared__ float2 cs[kRowK][kRowTile];
  const int p = blockIdx.x;
  const int box = a.box;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const float2* G = a.G + (long long)p * a.H * box;
  for (int yb0 = 0; yb0 < box; yb0 += kRowTile) {
    for (int xb0 = 0; xb0 < box; xb0 += kRowTile) {
      float acc[6][6];
#pragma unroll
      for (int i = 0; i < 6; i++)
#pragma unroll
        for (int j = 0; j < 6; j++) acc[i][j] = 0.f;
      for (int k0 = 0; k0 < a.H; k0 += kRowK) {
        __syncthreads();
        for (int t = threadIdx.x; t < kRowK * kRowTile; t += blockDim.x) {
          const int kk = t / kRowTile, c = t - kk * kRowTile;
          const int kx = k0 + kk;
          const bool okk = kx < a.H;
          gs[kk][c] = (okk && yb0 + c < box) ? G[(long long)kx * box + yb0 + c] : make_float2(0.f, 0.f);
          cs[kk][c] = (okk && xb0 + c < box) ? a.cs[(long long)kx * box + xb0 + c] : make_float2(0.f, 0.f);
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < kRowK; kk++) {
          float2 g[6], c[6];
#pragma unroll
          for (int i = 0; i < 6; i++) g[i] = gs[kk][ty + 16 * i];
#pragma unroll
          for (int j = 0; j < 6; j++) c[j] = cs[kk][tx + 16 * j];
#pragma unroll
          for (int i = 0; i < 6; i++)
#pragma unroll
            for (int j = 0; j < 6; j++) acc[i][j] = fmaf(g[i].x, c[j].x, fmaf(-g[i].y, c[j].y, acc[i][j]));
        }
      }
#pragma unroll
      for (int i = 0; i < 6; i++) {
        const int yb = yb0 + ty + 16 * i;
        if (yb >= box) continue;
#pragma unroll
        for (int j = 0; j < 6; j++) {
          const int xb = xb0 + tx + 16 * j;
          if (xb < box) a.boxes[((long long)p * box + yb) * box + xb] = acc[i][j];
        }
      }
    }
  }
}

cudaError_t launch_pair_rows(const PairRowsArgs& a, cudaStream_t st) {
  k_pair_rows<<<a.npairs, kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

// ==================================================================== peak ==
constexpr int kSub = 16;
constexpr int kPad = 512;
constexpr int kUp = 32;

struct PeakSmem {
  double2 g1[kPad][8];     // column-inverse of the masked sub-box spectrum
  double2 tw[kPad];        // exp(+2 pi i m / 512)
  double2 s[kSub][9];      // masked 16x16 half spectrum
  double2 rx[kSub][9];     // row transforms of the sub-box
  double sub[kSub][kSub];
  double rv[kThreads / 32];
  int ri[kThreads / 32];
  float fv[kThreads / 32];
  int fi[kThreads / 32];
  double f00;
};

size_t peak_smem() { return sizeof(PeakSmem); }

// (v, i) beats (bv, bi): larger value, or equal value and earlier scan index.
template <typename T>
__device__ __forceinline__ bool better(T v, int i, T bv, int bi) {
  return v > bv || (v == bv && i < bi);
}

__global__ void __launch_bounds__(kThreads) k_peak(PeakArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  PeakSmem& S = *reinterpret_cast<PeakSmem*>(smraw);
  const int p = blockIdx.x;
  const int box = a.box;
  const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, wid = tid >> 5;
  const float* bm = a.boxes + (long long)p * box * box;
  const int wnoise = a.nps - 1;
  const int hb = box / 2;

  // ---- integer peak (cufunc.cu:409-424): strict '>' from -1e9, y outer, x inner
  float bv = -1e9f;
  int bi = 0x7fffffff;
  for (int idx = tid; idx < box * box; idx += nth) {
    const int yy = idx / box, xx = idx - yy * box;
    if (abs(xx - hb) <= wnoise && abs(yy - hb) <= wnoise) continue;
    const float v = bm[idx];
    if (v > -1e9f && better(v, idx, bv, bi)) {
      bv = v;
      bi = idx;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (better(ov, oi, bv, bi)) {
      bv = ov;
      bi = oi;
    }
  }
  if (lane == 0) {
    S.fv[wid] = bv;
    S.fi[wid] = bi;
  }
  __syncthreads();
  bv = S.fv[0];
  bi = S.fi[0];
  for (int w = 1; w < nth / 32; w++)
    if (better(S.fv[w], S.fi[w], bv, bi)) {
      bv = S.fv[w];
      bi = S.fi[w];
    }
  int ix = 0, iy = 0;
  if (bi != 0x7fffffff) {
    iy = bi / box;
    ix = bi - iy * box;
  }
  int offx = ix - kSub / 2, offy = iy - kSub / 2;
  if (offx + kSub > box) offx = box - kSub;
  else if (offx < 0) offx = 0;
  if (offy + kSub > box) offy = box - kSub;
  else if (offy < 0) offy = 0;

  // ---- sub-box, tables
  for (int t = tid; t < kSub * kSub; t += nth) {
    const int yy = t / kSub, xx = t - yy * kSub;
    S.sub[yy][xx] = (double)bm[(offy + yy) * box + offx + xx];
  }
  for (int m = tid; m < kPad; m += nth) {
    double sn, cn;
    sincospi((double)m / (kPad / 2), &sn, &cn);
    S.tw[m] = make_double2(cn, sn);
  }
  __syncthreads();
  // R2C along x: rx[y][kx] = sum_x sub[y][x] exp(-2 pi i kx x / 16)
  for (int t = tid; t < kSub * 9; t += nth) {
    const int yy = t / 9, k = t - yy * 9;
    double re = 0.0, im = 0.0;
    for (int xx = 0; xx < kSub; xx++) {
      const double2 w = S.tw[((k * xx) & (kSub - 1)) * (kPad / kSub)];
      re += S.sub[yy][xx] * w.x;
      im -= S.sub[yy][xx] * w.y;
    }
    S.rx[yy][k] = make_double2(re, im);
  }
  __syncthreads();
  // along y, then the cosine mask (func.cpp:348-370)
  for (int t = tid; t < kSub * 9; t += nth) {
    const int j = t / 9, k = t - j * 9;
    double re = 0.0, im = 0.0;
    for (int yy = 0; yy < kSub; yy++) {
      const double2 w = S.tw[((j * yy) & (kSub - 1)) * (kPad / kSub)];  // exp(+i..)
      const double2 v = S.rx[yy][k];
      re += v.x * w.x + v.y * w.y;  // v * conj(w)
      im += v.y * w.x - v.x * w.y;
    }
    const double wt = a.w16[j * 9 + k];
    S.s[j][k] = make_double2(re * wt, im * wt);
  }
  __syncthreads();
  // zero-padded inverse along y: g1[Y][kx] = sum_j s[j][kx] exp(+2 pi i ky_j Y / 512)
  for (int t = tid; t < kPad * 8; t += nth) {
    const int Y = t >> 3, k = t & 7;
    double re = 0.0, im = 0.0;
    for (int j = 0; j < kSub; j++) {
      const int ky = j < kSub / 2 ? j : j - kSub;
      const double2 w = S.tw[(ky * Y) & (kPad - 1)];
      const double2 v = S.s[j][k];
      re += v.x * w.x - v.y * w.y;
      im += v.x * w.y + v.y * w.x;
    }
    S.g1[Y][k] = make_double2(re, im);
  }
  __syncthreads();
  // C2R along x on the 512 grid and the argmax (cufunc.cu:457-476)
  const int ox = (hb - offx) * kUp, oy = (hb - offy) * kUp, wns = kUp * wnoise;
  double best = -INFINITY;
  int bidx = 0x7fffffff;
  for (int X = tid; X < kPad; X += nth) {
    double2 c[8];
#pragma unroll
    for (int k = 1; k < 8; k++) c[k] = S.tw[(k * X) & (kPad - 1)];
    const bool xex = abs(X - ox) <= wns;
    for (int Y = 0; Y < kPad; Y++) {
      double f = S.g1[Y][0].x;
#pragma unroll
      for (int k = 1; k < 8; k++) {
        const double2 g = S.g1[Y][k];
        f += 2.0 * (g.x * c[k].x - g.y * c[k].y);
      }
      if (X == 0 && Y == 0) S.f00 = f;
      if (xex && abs(Y - oy) <= wns) continue;
      const int idx = Y * kPad + X;
      if (better(f, idx, best, bidx)) {
        best = f;
        bidx = idx;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
    if (better(ov, oi, best, bidx)) {
      best = ov;
      bidx = oi;
    }
  }
  __syncthreads();
  if (lane == 0) {
    S.rv[wid] = best;
    S.ri[wid] = bidx;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < nth / 32; w++)
      if (better(S.rv[w], S.ri[w], best, bidx)) {
        best = S.rv[w];
        bidx = S.ri[w];
      }
    int sxp = 0, syp = 0;
    double bestcc = S.f00;
    if (bidx != 0x7fffffff && best > S.f00) {
      sxp = bidx % kPad;
      syp = bidx / kPad;
      bestcc = best;
    }
    const float sx = (float)(offx + sxp / (double)kUp) - (float)hb;
    const float sy = (float)(offy + syp / (double)kUp) - (float)hb;
    a.shift[2 * p] = sx;
    a.shift[2 * p + 1] = sy;
    a.cc[p] = (float)(bestcc / a.n / a.n / kSub / kSub);
    a.peak[2 * p] = ix;
    a.peak[2 * p + 1] = iy;
  }
}

cudaError_t launch_peak(const PeakArgs& a, cudaStream_t st) {
  const size_t smem = peak_smem();
  cudaError_t e = allow_smem((const void*)k_peak, smem);
  if (e != cudaSuccess) return e;
  k_peak<<<a.npairs, kThreads, smem, st>>>(a);
  return cudaGetLastError();
}

// ============================================================== shift-sum ==
size_t shift_sum_smem(int n, int nsum) {
  return (size_t)3 * n * sizeof(float2) + (size_t)nsum * sizeof(float2);
}

__global__ void __launch_bounds__(kThreads) k_shift_sum(ShiftSumArgs a, const float2* __restrict__ ey) {
  extern __shared__ float2 sm[];
  const int n = a.n;
  float2* acc = sm;
  float2* b1 = sm + n;
  float2* tw = sm + 2 * n;
  float2* ex = sm + 3 * n;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int kx = blockIdx.x;
  if (a.mode == 1) copy_table(tw, a.tw, n);
  for (int f = tid; f < a.nsum; f += nth) {
    double sn, cn;
    // exp(+2 pi i sx kx / n), argument reduced in double
    const double t = a.shifts[f].x * (double)kx / (double)n;
    sincospi(2.0 * (t - rint(t)), &sn, &cn);
    ex[f] = make_float2((float)cn, (float)sn);
  }
  for (int ky = tid; ky < n; ky += nth) acc[ky] = make_float2(0.f, 0.f);
  __syncthreads();
  for (int f = 0; f < a.nsum; f++) {
    const float2* col = a.spec + (long long)a.frames[f] * a.stride + (long long)kx * a.ldn;
    const float2 e = ex[f];
    const float2* eyf = ey + (long long)f * n;
    const bool ap = a.apply[f] != 0;
    for (int ky = tid; ky < n; ky += nth) {
      float2 v = col[ky];
      if (ap) v = cmul(v, cmul(e, eyf[ky]));
      acc[ky] = cadd(acc[ky], v);
    }
  }
  __syncthreads();
  if (a.mode == 0) {
    for (int ky = tid; ky < n; ky += nth) a.out[(long long)kx * a.ld_out + ky] = acc[ky];
    return;
  }
  float2* X = fft_run<true, false>(acc, b1, a.plan, 1, n, tw, tid, nth);
  for (int y = tid; y < n; y += nth) a.out[(long long)y * a.ld_out + kx] = X[y];
}

// ============================================================ count sums ==
// One thread per 4 consecutive crop pixels of a row; frames summed in int32
// registers (exact: |pixel| <= 65535 and at most 2^15 frames).
template <typename Px>
__global__ void __launch_bounds__(kThreads) k_count_sum(CountSumArgs a) {
  const int per_row = (a.nu + 3) / 4;
  const long long total = (long long)per_row * a.nu;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(t / per_row);
    const int x0 = (int)(t - (long long)y * per_row) * 4;
    const int cnt = min(4, a.nu - x0);
    int acc[4] = {0, 0, 0, 0};
    const Px* base = reinterpret_cast<const Px*>(a.frames) + (long long)(a.offy + y) * a.nx + a.offx + x0;
    for (int f = a.first; f <= a.last; f++) {
      const Px* row = base + (long long)f * a.frame_pixels;
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (i < cnt) acc[i] += (int)row[i];
    }
    int* o = a.out + (long long)y * a.nu + x0;
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (i < cnt) o[i] = acc[i];
  }
}

cudaError_t launch_count_sum(const CountSumArgs& a, cudaStream_t st) {
  const long long items = (long long)((a.nu + 3) / 4) * a.nu;
  const int grid = (int)std::min<long long>((items + kThreads - 1) / kThreads, 148LL * 16);
  switch (a.mode) {
    case 0: k_count_sum<int8_t><<<grid, kThreads, 0, st>>>(a); break;
    case 1: k_count_sum<int16_t><<<grid, kThreads, 0, st>>>(a); break;
    case 6: k_count_sum<uint16_t><<<grid, kThreads, 0, st>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

__global__ void k_ramp(RampArgs a) {
  const int f = blockIdx.y;
  const double sy = a.shifts[f].y;
  for (int ky = blockIdx.x * blockDim.x + threadIdx.x; ky < a.n; ky += gridDim.x * blockDim.x) {
    const int y = ky < a.n / 2 ? ky : ky - a.n;
    const double t = sy * (double)y / (double)a.n;
    double sn, cn;
    sincospi(2.0 * (t - rint(t)), &sn, &cn);
    a.ey[(long long)f * a.n + ky] = make_float2((float)cn, (float)sn);
  }
}

// Two-level variant for columns of length N1*N2: each thread keeps the
// running sums of its E = ceil(n/256) column elements in registers, so a
// frame's column is requested with E independent loads per thread; the final
// inverse along ky is the two-level transform.
template <int N1, int N2>
__global__ void __launch_bounds__(kThreads) k_shift_sum2l(ShiftSumArgs a, const float2* __restrict__ ey) {
  using TL = TwoLevel<N1, N2>;
  constexpr int N = TL::N;
  constexpr int E = (N + kThreads - 1) / kThreads;
  extern __shared__ float2 sm2l[];
  float2* col = sm2l;         // accumulated column, then the step-A input
  float2* ysm = sm2l + N;     // exchange buffer
  float2* ex = sm2l + 2 * N;  // per-frame exp(+2 pi i sx kx / n)
  const int tid = threadIdx.x;
  const int kx = blockIdx.x;
  for (int f = tid; f < a.nsum; f += kThreads) {
    double sn, cn;
    const double t = a.shifts[f].x * (double)kx / (double)N;
    sincospi(2.0 * (t - rint(t)), &sn, &cn);
    ex[f] = make_float2((float)cn, (float)sn);
  }
  __syncthreads();
  float2 acc[E];
#pragma unroll
  for (int j = 0; j < E; j++) acc[j] = make_float2(0.f, 0.f);
  for (int f = 0; f < a.nsum; f++) {
    const float2* c = a.spec + (long long)a.frames[f] * a.stride + (long long)kx * a.ldn;
    const float2* eyf = ey + (long long)f * N;
    const float2 e = ex[f];
    const bool ap = a.apply[f] != 0;
#pragma unroll
    for (int j = 0; j < E; j++) {
      const int ky = tid + kThreads * j;
      if (ky < N) {
        float2 v = __ldg(c + ky);
        if (ap) v = cmul(v, cmul(e, __ldg(eyf + ky)));
        acc[j] = cadd(acc[j], v);
      }
    }
  }
  if (a.mode == 0) {
#pragma unroll
    for (int j = 0; j < E; j++) {
      const int ky = tid + kThreads * j;
      if (ky < N) a.out[(long long)kx * a.ld_out + ky] = acc[j];
    }
    return;
  }
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int ky = tid + kThreads * j;
    if (ky < N) col[ky] = acc[j];
  }
  __syncthreads();
  float2* out = a.out;
  const long long ld = a.ld_out;
  TL::template run<true, false>(ysm, a.tw, [&](int i) { return col[i]; },
                                [&](int k, float2 v) { out[(long long)k * ld + kx] = v; });
}

cudaError_t launch_shift_sum(const ShiftSumArgs& a, float2* ey, cudaStream_t st) {
  RampArgs r;
  r.shifts = a.shifts;
  r.nsum = a.nsum;
  r.n = a.n;
  r.ey = ey;
  dim3 g((a.n + 255) / 256, a.nsum);
  k_ramp<<<g, 256, 0, st>>>(r);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int n1 = 0, n2 = 0;
  if (two_level_split(a.n, n1, n2)) {
    const size_t smem2 = (size_t)(2 * a.n + a.nsum) * sizeof(float2);
#define MC_TL_SUM(A, B)                                                                                       \
  if (n1 == (A) && n2 == (B)) {                                                                               \
    e = allow_smem((const void*)k_shift_sum2l<A, B>, smem2);                                                \
    if (e != cudaSuccess) return e;                                                                           \
    k_shift_sum2l<A, B><<<a.H, kThreads, smem2, st>>>(a, ey);                                                 \
    return cudaGetLastError();                                                                                \
  }
    MC_TWO_LEVEL_LIST(MC_TL_SUM)
#undef MC_TL_SUM
  }
  const size_t smem = shift_sum_smem(a.n, a.nsum);
  e = allow_smem((const void*)k_shift_sum, smem);
  if (e != cudaSuccess) return e;
  k_shift_sum<<<a.H, kThreads, smem, st>>>(a, ey);
  return cudaGetLastError();
}

// ================================================================ C2R rows ==
size_t c2r_rows_smem(int n) { return (size_t)3 * n * sizeof(float2); }

__global__ void __launch_bounds__(kThreads) k_c2r_rows(C2rRowsArgs a) {
  extern __shared__ float2 sm[];
  const int n = a.n, H = a.H, half = n / 2;
  float2* b0 = sm;
  float2* b1 = sm + n;
  float2* tw = sm + 2 * n;
  copy_table(tw, a.tw, n);
  const int tid = threadIdx.x, nth = blockDim.x;
  const int y0 = 2 * blockIdx.x, y1 = y0 + 1;
  const float2* g0 = a.t2 + (long long)y0 * a.ld_t2;
  const float2* g1 = a.t2 + (long long)y1 * a.ld_t2;
  for (int k = tid; k < n; k += nth) {
    float2 u, v;
    if (k <= half) {
      u = g0[k];
      v = g1[k];
      if (k == 0 || k == half) {  // C2R uses only the real part of DC and Nyquist
        u.y = 0.f;
        v.y = 0.f;
      }
    } else {
      u = g0[n - k];
      v = g1[n - k];
      u.y = -u.y;
      v.y = -v.y;
    }
    b0[k] = make_float2(u.x - v.y, u.y + v.x);  // u + i v
  }
  (void)H;
  __syncthreads();
  float2* X = fft_run<true, false>(b0, b1, a.plan, 1, n, tw, tid, nth);
  for (int x = tid; x < n; x += nth) {
    const float2 z = X[x];
    a.image[(long long)y0 * n + x] = z.x * a.scale;
    a.image[(long long)y1 * n + x] = z.y * a.scale;
  }
}

// =============================================================== adjoint ==
template <int E>
__global__ void __launch_bounds__(kThreads) k_objective(ObjectiveArgs a) {
  extern __shared__ double smo[];
  double* red = smo;                                                   // [warps][5]
  float2* ex = reinterpret_cast<float2*>(smo + (kThreads / 32) * 5);  // [nframes]
  const int n = a.n, half = n / 2;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int kx = blockIdx.x;
  const float h = (kx == 0 || kx == half) ? 1.f : 2.f;
  const float ox = 6.283185307179586f * (float)kx / (float)n;
  for (int f = tid; f < a.nframes; f += kThreads) {
    double sn, cn;
    const double t = a.shifts[f].x * (double)kx / (double)n;
    sincospi(2.0 * (t - rint(t)), &sn, &cn);
    ex[f] = make_float2((float)cn, (float)sn);
  }
  float2 s[E];
  float hw[E], oy[E];
  double jsum = 0.0;
  const float2* Scol = a.S + (long long)kx * a.ldn;
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int ky = tid + kThreads * j;
    if (ky < n) {
      const int y = ky < half ? ky : ky - n;
      s[j] = __ldg(Scol + ky);
      hw[j] = h * expf(a.mbf * (float)(kx * kx + y * y));
      oy[j] = 6.283185307179586f * (float)y / (float)n;
      jsum += (double)(hw[j] * (s[j].x * s[j].x + s[j].y * s[j].y));
    } else {
      s[j] = make_float2(0.f, 0.f);
      hw[j] = 0.f;
      oy[j] = 0.f;
    }
  }
  __syncthreads();
  // J partial
  for (int o = 16; o > 0; o >>= 1) jsum += __shfl_xor_sync(0xffffffffu, jsum, o);
  if (lane == 0) red[wid * 5] = jsum;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; w++) t += red[w * 5];
    a.partialJ[kx] = t;
  }
  __syncthreads();
  for (int f = 0; f < a.nframes; f++) {
    const float2* c = a.spec + (long long)f * a.stride + (long long)kx * a.ldn;
    const float2* eyf = a.ey + (long long)f * n;
    const float2 e = ex[f];
    double gx = 0, gy = 0, hxx = 0, hxy = 0, hyy = 0;
#pragma unroll
    for (int j = 0; j < E; j++) {
      const int ky = tid + kThreads * j;
      if (ky < n) {
        const float2 P = cmul(__ldg(c + ky), cmul(e, __ldg(eyf + ky)));
        const float2 d = csub(s[j], P);
        const float2 u = cmulc(P, d);  // conj(d) * P
        const double wi = (double)(hw[j] * u.y), wr = (double)(hw[j] * u.x);
        const double y = (double)oy[j];
        gx += wi;
        gy += wi * y;
        hxx += wr;
        hxy += wr * y;
        hyy += wr * y * y;
      }
    }
    // omega_x is constant over the column: apply it after the sums
    double v[5] = {gx * ox, gy, hxx * ox * ox, hxy * ox, hyy};
#pragma unroll
    for (int q = 0; q < 5; q++)
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < 5; q++) red[wid * 5 + q] = v[q];
    __syncthreads();
    if (tid < 5) {
      double t = 0.0;
      for (int w = 0; w < kThreads / 32; w++) t += red[w * 5 + tid];
      a.partial[((long long)kx * a.nframes + f) * 5 + tid] = t;
    }
    __syncthreads();
  }
}

// Column partials -> per-frame totals in a fixed order (deterministic).
__global__ void k_objective_reduce(ObjectiveArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nv = a.nframes * 5;
  if (t < nv) {
    double acc = 0.0;
    for (int kx = 0; kx < a.H; kx++) acc += a.partial[(long long)kx * nv + t];
    a.out[t] = -2.0 * acc;
  } else if (t == nv) {
    double acc = 0.0;
    for (int kx = 0; kx < a.H; kx++) acc += a.partialJ[kx];
    a.out[nv] = acc;
  }
}

cudaError_t launch_ramp(const double2* shifts, int nsum, int n, float2* ey, cudaStream_t st) {
  RampArgs r;
  r.shifts = shifts;
  r.nsum = nsum;
  r.n = n;
  r.ey = ey;
  dim3 g((n + 255) / 256, nsum);
  k_ramp<<<g, 256, 0, st>>>(r);
  return cudaGetLastError();
}

cudaError_t launch_objective(const ObjectiveArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(double) * (kThreads / 32) * 5 + sizeof(float2) * (size_t)a.nframes;
  cudaError_t e;
  const int E = (a.n + kThreads - 1) / kThreads;
  if (E <= 8) {
    e = allow_smem((const void*)k_objective<8>, smem);
    if (e != cudaSuccess) return e;
    k_objective<8><<<a.H, kThreads, smem, st>>>(a);
  } else if (E <= 16) {
    e = allow_smem((const void*)k_objective<16>, smem);
    if (e != cudaSuccess) return e;
    k_objective<16><<<a.H, kThreads, smem, st>>>(a);
  } else if (E <= 36) {
    e = allow_smem((const void*)k_objective<36>, smem);
    if (e != cudaSuccess) return e;
    k_objective<36><<<a.H, kThreads, smem, st>>>(a);
  } else {
    return cudaErrorInvalidValue;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int nv = a.nframes * 5 + 1;
  k_objective_reduce<<<(nv + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

// Two-level variant: rows y, y+1 packed as Z = G_y + i G_{y+1} with the
// Hermitian extension formed in the load (real DC and Nyquist).
template <int N1, int N2>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T) k_c2r_rows2l(C2rRowsArgs a) {
  using TL = TwoLevel<N1, N2>;
  constexpr int N = TL::N;
  __shared__ float2 ysm[N];
  const int y0 = 2 * blockIdx.x, y1 = y0 + 1;
  const float2* g0 = a.t2 + (long long)y0 * a.ld_t2;
  const float2* g1 = a.t2 + (long long)y1 * a.ld_t2;
  float* i0 = a.image + (long long)y0 * N;
  float* i1 = a.image + (long long)y1 * N;
  const float sc = a.scale;
  TL::template run<true, false>(
      ysm, a.tw,
      [&](int k) {
        float2 u, v;
        if (k <= N / 2) {
          u = __ldg(g0 + k);
          v = __ldg(g1 + k);
          if (k == 0 || k == N / 2) {
            u.y = 0.f;
            v.y = 0.f;
          }
        } else {
          u = __ldg(g0 + N - k);
          v = __ldg(g1 + N - k);
          u.y = -u.y;
          v.y = -v.y;
        }
        return make_float2(u.x - v.y, u.y + v.x);
      },
      [&](int x, float2 z) {
        i0[x] = z.x * sc;
        i1[x] = z.y * sc;
      });
}

cudaError_t launch_c2r_rows(const C2rRowsArgs& a, cudaStream_t st) {
  int n1 = 0, n2 = 0;
  if (two_level_split(a.n, n1, n2)) {
#define MC_TL_C2R(A, B)                                              \
  if (n1 == (A) && n2 == (B)) {                                      \
    k_c2r_rows2l<A, B><<<a.n / 2, TwoLevel<A, B>::T, 0, st>>>(a);    \
    return cudaGetLastError();                                       \
  }
    MC_TWO_LEVEL_LIST(MC_TL_C2R)
#undef MC_TL_C2R
  }
  const size_t smem = c2r_rows_smem(a.n);
  cudaError_t e = allow_smem((const void*)k_c2r_rows, smem);
  if (e != cudaSuccess) return e;
  k_c2r_rows<<<a.n / 2, kThreads, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mc
