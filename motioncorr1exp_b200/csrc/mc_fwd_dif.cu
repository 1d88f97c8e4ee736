// Forward transforms of libmc for lengths 2N with a two-level N (sm_100a):
// 7420 = 2 x 3710 at -bin 2 (DFAlign.cu:710-806, cufunc.cu:162-176).
#include <algorithm>

#include "kcommon.cuh"

namespace mc {

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
      case MC_MODE_U8: MC_DIF_RAW(A, B, uint8_t)                                                      \
      case 1: MC_DIF_RAW(A, B, int16_t)                                                               \
      case 6: MC_DIF_RAW(A, B, uint16_t)                                                              \
      case MC_MODE_F16: MC_DIF_RAW(A, B, __half)                                                      \
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

}  // namespace mc
