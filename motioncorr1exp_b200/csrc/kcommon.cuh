// Device code shared by the kernel translation units of libmc (mc_fwd*.cu,
// mc_pair.cu, mc_sum.cu): constants, pixel decode, the two-level register FFT
// and the raw-row staging helpers.
#pragma once
#include <cuda_fp16.h>
#include <math.h>
#include <stdint.h>

#include "kernels.cuh"
#include "codelets_gen.cuh"

namespace mc {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float load_pixel(const void* frame, int mode, long long idx) {
  switch (mode) {
    case 0: return (float)((const int8_t*)frame)[idx];
    case MC_MODE_U8: return (float)((const uint8_t*)frame)[idx];
    case 1: return (float)((const int16_t*)frame)[idx];
    case 6: return (float)((const uint16_t*)frame)[idx];
    case MC_MODE_F16: return __half2float(((const __half*)frame)[idx]);
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

// Built-in radix-53 schedules of the forward row / column transforms: two
// output pairs per loop pass in both (measured on c2: the row pass 9 %
// faster paired; the column pass 12 % faster paired once its stores lost
// the crop test and the scale, 27 % slower before); a schedule
// (mc_schedule_set, the autotuner) can pick either.
constexpr bool kFwdRowsPaired = true;
constexpr bool kFwdColsPaired = true;
// Resident CTAs per SM the two-level transforms are compiled for (register cap).
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
                             int kmax = (N1 - 1) / 2, int lt_team = -1) {
    static_assert(T >= N2, "one k2 per thread");
    // lt_team: the thread's index in its team of T when a CTA runs several
    // transforms side by side (every team takes the same barriers)
    const int lt = lt_team >= 0 ? lt_team : (int)threadIdx.x;
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


// Two-level splits compiled in (N1, N2).
#define MC_TWO_LEVEL_LIST(X) X(53, 70) X(64, 64) X(32, 64) X(32, 32) X(16, 16) X(16, 32)
bool two_level_split(int n, int& n1, int& n2);

}  // namespace mc
