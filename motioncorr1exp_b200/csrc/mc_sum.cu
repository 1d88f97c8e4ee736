// Peak search, sum and adjoint kernels of libmc (sm_100a): integer peak and
// x32 Fourier-upsampled sub-pixel peak (cufunc.cu:396-497), phase-shift-and-
// accumulate with the inverse column FFT (cufunc.cu:372-393), final C2R rows
// (DFAlign.cu:1287-1292), exact count sums and the objective of the gradient
// refinement.
#include <algorithm>

#include "kcommon.cuh"

namespace mc {

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
    case MC_MODE_U8: k_count_sum<uint8_t><<<grid, kThreads, 0, st>>>(a); break;
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

// Accumulation alone (no transform): each CTA covers kSumChunk consecutive ky
// of one kx column, kSumE per thread, with the operations and frame order of
// the fused kernels, so the sum spectrum is bitwise the same.  The loads of
// kSumG frames are issued before their products are added: 64 registers,
// four CTAs per SM and 2 * kSumE * kSumG loads per thread in flight, where
// the fused two-level kernel (its transform needs most of the register file)
// runs one CTA per SM.  Measured on 3710^2 x 40 frames: 0.38 ms against a
// 0.34 ms HBM floor (kSumG = 1: 0.56 ms; kSumE = 2 or 8: slower).
constexpr int kSumE = 4;
constexpr int kSumG = 2;
constexpr int kSumChunk = kThreads * kSumE;

__global__ void __launch_bounds__(kThreads) k_shift_acc(ShiftSumArgs a, const float2* __restrict__ ey,
                                                        float2* out, long long ld_out) {
  extern __shared__ float2 exs[];  // per-frame exp(+2 pi i sx kx / n)
  const int tid = threadIdx.x, kx = blockIdx.y, n = a.n;
  for (int f = tid; f < a.nsum; f += kThreads) {
    double sn, cn;
    const double t = a.shifts[f].x * (double)kx / (double)n;
    sincospi(2.0 * (t - rint(t)), &sn, &cn);
    exs[f] = make_float2((float)cn, (float)sn);
  }
  __syncthreads();
  const int k0 = blockIdx.x * kSumChunk + tid;
  float2 acc[kSumE];
#pragma unroll
  for (int j = 0; j < kSumE; j++) {
    const int ky = k0 + kThreads * j;
    acc[j] = (a.accumulate && ky < n) ? out[(long long)kx * ld_out + ky] : make_float2(0.f, 0.f);
  }
  const float2* colx = a.spec + (long long)kx * a.ldn;
  for (int f0 = 0; f0 < a.nsum; f0 += kSumG) {
    float2 v[kSumG][kSumE], y[kSumG][kSumE];
    bool ap[kSumG];
#pragma unroll
    for (int g = 0; g < kSumG; g++) {
      const int f = f0 + g;
      ap[g] = f < a.nsum && a.apply[f] != 0;
      if (f < a.nsum) {
        const float2* c = colx + (long long)a.frames[f] * a.stride;
        const float2* eyf = ey + (long long)f * n;
#pragma unroll
        for (int j = 0; j < kSumE; j++) {
          const int ky = k0 + kThreads * j;
          if (ky < n) {
            v[g][j] = __ldg(c + ky);
            if (ap[g]) y[g][j] = __ldg(eyf + ky);
          }
        }
      }
    }
#pragma unroll
    for (int g = 0; g < kSumG; g++) {
      const int f = f0 + g;
      if (f < a.nsum) {
        const float2 e = exs[f];
#pragma unroll
        for (int j = 0; j < kSumE; j++) {
          float2 w = v[g][j];
          if (ap[g]) w = cmul(w, cmul(e, y[g][j]));
          acc[j] = cadd(acc[j], w);
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kSumE; j++) {
    const int ky = k0 + kThreads * j;
    if (ky < n) out[(long long)kx * ld_out + ky] = acc[j];
  }
}

// The inverse along ky of each accumulated column, written transposed
// (out[y * ld_out + kx]) for the C2R row pass: the transform of the fused
// two-level kernel, here at TwoLevel's own CTA size.
template <int N1, int N2>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS)
    k_sum_cols2l(const float2* __restrict__ in, long long ld_in, const float2* __restrict__ tw, float2* out,
                 long long ld_out) {
  using TL = TwoLevel<N1, N2>;
  __shared__ float2 ysm[TL::N];
  const int kx = blockIdx.x;
  const float2* col = in + (long long)kx * ld_in;
  TL::template run<true, false>(ysm, tw, [&](int i) { return __ldg(col + i); },
                                [&](int k, float2 v) { out[(long long)k * ld_out + kx] = v; });
}

cudaError_t launch_shift_acc(const ShiftSumArgs& a, const float2* ey, float2* out, long long ld_out,
                             cudaStream_t st) {
  const size_t smem = (size_t)a.nsum * sizeof(float2);
  cudaError_t e = allow_smem((const void*)k_shift_acc, smem);
  if (e != cudaSuccess) return e;
  dim3 g((a.n + kSumChunk - 1) / kSumChunk, a.H);
  k_shift_acc<<<g, kThreads, smem, st>>>(a, ey, out, ld_out);
  return cudaGetLastError();
}

int shift_sum_kernels(const ShiftSumArgs& a) {
  int n1, n2;
  return (a.mode == 1 && a.acc && two_level_split(a.n, n1, n2)) ? 3 : 2;  // k_ramp first
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
  if (a.mode == 0) return launch_shift_acc(a, ey, a.out, a.ld_out, st);
  int n1 = 0, n2 = 0;
  if (a.acc && two_level_split(a.n, n1, n2)) {
    e = launch_shift_acc(a, ey, a.acc, a.ldn, st);
    if (e != cudaSuccess) return e;
#define MC_TL_COLS(A, B)                                                                     \
  if (n1 == (A) && n2 == (B)) {                                                              \
    k_sum_cols2l<A, B><<<a.H, TwoLevel<A, B>::T, 0, st>>>(a.acc, a.ldn, a.tw, a.out, a.ld_out); \
    return cudaGetLastError();                                                               \
  }
    MC_TWO_LEVEL_LIST(MC_TL_COLS)
#undef MC_TL_COLS
  }
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
// Each thread's per-frame partials over its E <= 36 column elements add in
// FP32 (the terms themselves are FP32 products): five conversions per frame
// instead of three per element; warps and columns add in FP64.  The column
// loads go out in batches of eight spectrum and eight ramp values before any
// is used (issued one by one, each waited for its own latency: 3.3 ms per
// call at 4096^2 x 60 frames, batched 2.2 ms).
//
// STAGE (E = 16): the column's S, weight and frequency terms live in shared
// memory ([j][thread], each thread reading only its own entries) instead of
// registers, and the loads are software-pipelined: the 16 elements a thread
// in two halves of eight, the next half's spectrum and ramp loads in flight
// while the current half is summed, across frames too (two CTAs per SM; at
// 4096^2 x 60 frames 1.50 -> 0.98 ms per call, bitwise the same).
// Each frame's five warp totals come from a reduce-scatter over the lanes
// (nine FP64 shuffles instead of twenty-five, the same addition tree).
template <int E, bool STAGE>
__device__ __forceinline__ void objective_body(const ObjectiveArgs& a) {
  constexpr int W = kThreads / 32;
  constexpr int KB = STAGE ? E : (E < 8 ? E : 8);
  constexpr int R = STAGE ? 1 : E;  // register copies of the column terms
  extern __shared__ double smo[];
  double* red = smo;                                                          // [warps][5] (J)
  double* fred = smo + W * 5;                                                 // [nframes][warps][5]
  float2* ex = reinterpret_cast<float2*>(fred + (size_t)a.nframes * W * 5);  // [nframes]
  float2* ss = ex + a.nframes;                                                // [E][kThreads] (STAGE)
  float* shw = reinterpret_cast<float*>(ss + (STAGE ? E * kThreads : 0));     // [E][kThreads]
  float* soy = shw + (STAGE ? E * kThreads : 0);                              // [E][kThreads]
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
  float2 s[R];
  float hw[R], oy[R];
  double jsum = 0.0;
  const float2* Scol = a.S + (long long)kx * a.ldn;
#pragma unroll
  for (int j = 0; j < E; j++) {
    const int ky = tid + kThreads * j;
    float2 sv = make_float2(0.f, 0.f);
    float hv = 0.f, ov = 0.f;
    if (ky < n) {
      const int y = ky < half ? ky : ky - n;
      sv = __ldg(Scol + ky);
      hv = h * expf(a.mbf * (float)(kx * kx + y * y));
      ov = 6.283185307179586f * (float)y / (float)n;
      jsum += (double)(hv * (sv.x * sv.x + sv.y * sv.y));
    }
    if constexpr (STAGE) {
      ss[j * kThreads + tid] = sv;
      shw[j * kThreads + tid] = hv;
      soy[j * kThreads + tid] = ov;
    } else {
      s[j] = sv;
      hw[j] = hv;
      oy[j] = ov;
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
  // per frame: warp sums into shared memory, one barrier for all frames
  auto frame_sums = [&](int f, double* v) {
    // the five warp totals of frame f: lane (bits 4, 3, 2) = slot 4 b4 + 2 b3 + b2
    // receives slot's total after a reduce-scatter (nine shuffles for five values)
    double w[8] = {v[0], v[1], v[2], v[3], v[4], 0.0, 0.0, 0.0};
    const bool u4 = lane & 16, u3 = lane & 8, u2 = lane & 4;
    double x4[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const double send = u4 ? w[i] : w[i + 4];
      x4[i] = (u4 ? w[i + 4] : w[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    double x2[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const double send = u3 ? x4[i] : x4[i + 2];
      x2[i] = (u3 ? x4[i + 2] : x4[i]) + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    double x1 = (u2 ? x2[1] : x2[0]) + __shfl_xor_sync(0xffffffffu, u2 ? x2[0] : x2[1], 4);
    x1 += __shfl_xor_sync(0xffffffffu, x1, 2);
    x1 += __shfl_xor_sync(0xffffffffu, x1, 1);
    const int slot = (u4 ? 4 : 0) + (u3 ? 2 : 0) + (u2 ? 1 : 0);
    if ((lane & 3) == 0 && slot < 5) fred[((size_t)f * W + wid) * 5 + slot] = x1;
  };
  if constexpr (STAGE && E == 16) {
    // software-pipelined: the column's 16 elements a thread in two halves of
    // eight, the next half's spectrum and ramp loads in flight while the
    // current half is summed (across frames too)
    constexpr int HB = 8;
    float2 pa[HB], qa[HB], pb[HB], qb[HB];
    auto colp = [&](int f) {
      return a.spec + (long long)(a.frames ? a.frames[f] : f) * a.stride + (long long)kx * a.ldn;
    };
#define MC_OBJ_LOAD(F, HH, P, Q)                            \
  {                                                         \
    const float2* c_ = colp(F);                             \
    const float2* e_ = a.ey + (long long)(F) * n;           \
    _Pragma("unroll") for (int b = 0; b < HB; b++) {        \
      const int ky = tid + kThreads * ((HH) * HB + b);      \
      if (ky < n) {                                         \
        P[b] = __ldg(c_ + ky);                              \
        Q[b] = __ldg(e_ + ky);                              \
      }                                                     \
    }                                                       \
  }
#define MC_OBJ_SUM(F, HH, P, Q)                                   \
  {                                                               \
    const float2 e = ex[F];                                       \
    _Pragma("unroll") for (int b = 0; b < HB; b++) {              \
      const int j = (HH) * HB + b;                                \
      const int ky = tid + kThreads * j;                          \
      if (ky < n) {                                               \
        const float2 sj = ss[j * kThreads + tid];                 \
        const float hj = shw[j * kThreads + tid];                 \
        const float y = soy[j * kThreads + tid];                  \
        const float2 P_ = cmul(P[b], cmul(e, Q[b]));              \
        const float2 d = csub(sj, P_);                            \
        const float2 u = cmulc(P_, d);                            \
        const float wi = hj * u.y, wr = hj * u.x;                 \
        fx += wi;                                                 \
        fy = fmaf(wi, y, fy);                                     \
        fxx += wr;                                                \
        fxy = fmaf(wr, y, fxy);                                   \
        fyy = fmaf(wr * y, y, fyy);                               \
      }                                                           \
    }                                                             \
  }
    if (a.nframes > 0) MC_OBJ_LOAD(0, 0, pa, qa)
    for (int f = 0; f < a.nframes; f++) {
      MC_OBJ_LOAD(f, 1, pb, qb)
      float fx = 0.f, fy = 0.f, fxx = 0.f, fxy = 0.f, fyy = 0.f;
      MC_OBJ_SUM(f, 0, pa, qa)
      if (f + 1 < a.nframes) MC_OBJ_LOAD(f + 1, 0, pa, qa)
      MC_OBJ_SUM(f, 1, pb, qb)
      const double gx = fx, gy = fy, hxx = fxx, hxy = fxy, hyy = fyy;
      double v[5] = {gx * ox, gy, hxx * ox * ox, hxy * ox, hyy};
      frame_sums(f, v);
    }
#undef MC_OBJ_LOAD
#undef MC_OBJ_SUM
  } else {
  for (int f = 0; f < a.nframes; f++) {
    const float2* c = a.spec + (long long)(a.frames ? a.frames[f] : f) * a.stride + (long long)kx * a.ldn;
    const float2* eyf = a.ey + (long long)f * n;
    const float2 e = ex[f];
    // loads in batches of KB spectrum + KB ramp values, all issued before use
    float fx = 0.f, fy = 0.f, fxx = 0.f, fxy = 0.f, fyy = 0.f;
#pragma unroll
    for (int j0 = 0; j0 < E; j0 += KB) {
      float2 pv[KB], qv[KB];
#pragma unroll
      for (int b = 0; b < KB; b++) {
        const int ky = tid + kThreads * (j0 + b);
        if (j0 + b < E && ky < n) {
          pv[b] = __ldg(c + ky);
          qv[b] = __ldg(eyf + ky);
        }
      }
#pragma unroll
      for (int b = 0; b < KB; b++) {
        const int j = j0 + b;
        const int ky = tid + kThreads * j;
        if (j < E && ky < n) {
          float2 sj;
          float hj, y;
          if constexpr (STAGE) {
            sj = ss[j * kThreads + tid];
            hj = shw[j * kThreads + tid];
            y = soy[j * kThreads + tid];
          } else {
            sj = s[j];
            hj = hw[j];
            y = oy[j];
          }
          const float2 P = cmul(pv[b], cmul(e, qv[b]));
          const float2 d = csub(sj, P);
          const float2 u = cmulc(P, d);  // conj(d) * P
          const float wi = hj * u.y, wr = hj * u.x;
          fx += wi;
          fy = fmaf(wi, y, fy);
          fxx += wr;
          fxy = fmaf(wr, y, fxy);
          fyy = fmaf(wr * y, y, fyy);
        }
      }
    }
    const double gx = fx, gy = fy, hxx = fxx, hxy = fxy, hyy = fyy;
    // omega_x is constant over the column: apply it after the sums
    double v[5] = {gx * ox, gy, hxx * ox * ox, hxy * ox, hyy};
    frame_sums(f, v);
  }
  }
  __syncthreads();
  for (int i = tid; i < a.nframes * 5; i += kThreads) {
    const int f = i / 5, q = i - f * 5;
    double t = 0.0;
    for (int w = 0; w < W; w++) t += fred[((size_t)f * W + w) * 5 + q];
    a.partial[((long long)kx * a.nframes + f) * 5 + q] = t;
  }
}

template <int E>
__global__ void __launch_bounds__(kThreads) k_objective(ObjectiveArgs a) {
  objective_body<E, false>(a);
}

__global__ void __launch_bounds__(kThreads, 2) k_objective_staged(ObjectiveArgs a) { objective_body<16, true>(a); }

// Column partials -> per-frame totals in a fixed order (deterministic): one
// CTA per total, each thread a strided run of columns, then a fixed tree.
constexpr int kReduceThreads = 256;
__global__ void __launch_bounds__(kReduceThreads) k_objective_reduce(ObjectiveArgs a) {
  __shared__ double part[kReduceThreads];
  const int t = blockIdx.x, nv = a.nframes * 5;
  double acc = 0.0;
  if (t < nv) {
    for (int kx = threadIdx.x; kx < a.H; kx += kReduceThreads) acc += a.partial[(long long)kx * nv + t];
  } else {
    for (int kx = threadIdx.x; kx < a.H; kx += kReduceThreads) acc += a.partialJ[kx];
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.out[t] = t < nv ? -2.0 * part[0] : part[0];
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
  const size_t smem = sizeof(double) * (kThreads / 32) * 5 * (1 + (size_t)a.nframes) +
                      sizeof(float2) * (size_t)a.nframes;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;  // more than ~600 frames
  cudaError_t e = cudaSuccess;
  const int E = (a.n + kThreads - 1) / kThreads;
  // staged column terms: 16 bytes per element; used while two CTAs fit an SM
  const size_t smem_st = smem + (size_t)16 * kThreads * 16;
  if (E > 8 && E <= 16 && smem_st <= 110 * 1024) {
    e = allow_smem((const void*)k_objective_staged, smem_st);
    if (e != cudaSuccess) return e;
    k_objective_staged<<<a.H, kThreads, smem_st, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_objective_reduce<<<a.nframes * 5 + 1, kReduceThreads, 0, st>>>(a);
    return cudaGetLastError();
  }
#define MC_OBJ(EE)                                                          \
  {                                                                         \
    e = allow_smem((const void*)k_objective<EE>, smem);                     \
    if (e != cudaSuccess) return e;                                         \
    k_objective<EE><<<a.H, kThreads, smem, st>>>(a);                        \
  }
  if (E <= 8) MC_OBJ(8)
  else if (E <= 16) MC_OBJ(16)
  else if (E <= 36) MC_OBJ(36)
  else return cudaErrorInvalidValue;
#undef MC_OBJ
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_objective_reduce<<<a.nframes * 5 + 1, kReduceThreads, 0, st>>>(a);
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

// ============================================================= quick-look ==
__global__ void k_ql_logmod(const float2* __restrict__ spec, int ldn, int n, float scale, float* __restrict__ img) {
  const int h = n / 2;
  const long long total = (long long)n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int r = (int)(t / n), c = (int)(t - (long long)r * n);
    if (c < h) {  // mirrored half (FFTModulusToDispBuf), row 0 repeats row 1
      if (r == 0) r = 1;
      r = n - r;
      c = n - c;
    }
    const int kx = c - h;
    const int ky = r >= h ? r - h : r + h;
    const float2 v = spec[(long long)kx * ldn + ky];
    img[t] = logf(1.f + sqrtf(v.x * v.x + v.y * v.y) * scale);
  }
}

__global__ void k_ql_crop(const float2* __restrict__ spec, int ldn, int n, int d, float2* __restrict__ out) {
  const int hd = d / 2;
  const int total = (hd + 1) * d;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int kx = t / d, k = t - kx * d;
    const int ky = k < hd ? k : n - d + k;
    out[t] = spec[(long long)kx * ldn + ky];
  }
}

// exp(+2 pi i m / d), m < d, into shared memory (one table per block)
__device__ __forceinline__ void ql_table(float2* tw, int d) {
  for (int m = threadIdx.x; m < d; m += blockDim.x) {
    double sn, cn;
    sincospi(2.0 * (double)m / (double)d, &sn, &cn);
    tw[m] = make_float2((float)cn, (float)sn);
  }
  __syncthreads();
}

// pass 1: tmp[kx][y] = sum_ky in[kx][ky] exp(+2 pi i ky y / d)
__global__ void k_ql_c2r_cols(const float2* __restrict__ in, int d, float2* __restrict__ tmp) {
  extern __shared__ float2 qtw[];
  ql_table(qtw, d);
  const int kx = blockIdx.x;
  const float2* row = in + (long long)kx * d;
  for (int y = threadIdx.x; y < d; y += blockDim.x) {
    float re = 0.f, im = 0.f;
    int e = 0;
    for (int ky = 0; ky < d; ky++) {
      const float2 w = qtw[e];
      const float2 v = row[ky];
      re += v.x * w.x - v.y * w.y;
      im += v.x * w.y + v.y * w.x;
      e += y;
      if (e >= d) e -= d;
    }
    tmp[(long long)kx * d + y] = make_float2(re, im);
  }
}

// pass 2: img[y][x] = scale * sum_kx h(kx) Re(tmp[kx][y] exp(+2 pi i kx x / d))
__global__ void k_ql_c2r_rows(const float2* __restrict__ tmp, int d, float scale, float* __restrict__ img) {
  extern __shared__ float2 qtw[];
  ql_table(qtw, d);
  const int y = blockIdx.x, hd = d / 2;
  for (int x = threadIdx.x; x < d; x += blockDim.x) {
    float acc = 0.f;
    int e = 0;
    for (int kx = 0; kx <= hd; kx++) {
      const float2 w = qtw[e];
      const float2 v = tmp[(long long)kx * d + y];
      const float h = (kx == 0 || kx == hd) ? 1.f : 2.f;
      acc += h * (v.x * w.x - v.y * w.y);
      e += x;
      if (e >= d) e -= d;
    }
    img[(long long)y * d + x] = acc * scale;
  }
}

cudaError_t launch_ql_logmod(const float2* spec, int ldn, int n, float scale, float* img, cudaStream_t st) {
  k_ql_logmod<<<148 * 8, 256, 0, st>>>(spec, ldn, n, scale, img);
  return cudaGetLastError();
}

cudaError_t launch_ql_crop(const float2* spec, int ldn, int n, int d, float2* out, cudaStream_t st) {
  k_ql_crop<<<(((d / 2 + 1) * d) + 255) / 256, 256, 0, st>>>(spec, ldn, n, d, out);
  return cudaGetLastError();
}

cudaError_t launch_ql_c2r(const float2* in, int d, float scale, float2* tmp, float* img, cudaStream_t st) {
  if (d > 4096) return cudaErrorInvalidValue;
  const size_t sm = sizeof(float2) * (size_t)d;
  k_ql_c2r_cols<<<d / 2 + 1, 256, sm, st>>>(in, d, tmp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_ql_c2r_rows<<<d, 256, sm, st>>>(tmp, d, scale, img);
  return cudaGetLastError();
}

}  // namespace mc
