// Forward row pass of libmc for two-level lengths (sm_100a): two rows packed
// as one complex FFT, raw-pixel staging when no dark/gain references apply
// (DFAlign.cu:710-806).
#include <algorithm>

#include "kcommon.cuh"

namespace mc {

// Forward rows without references, four rows per CTA: the rows are staged
// as raw pixels (a quarter of the float staging for 8-bit frames) and
// decoded in the step-A loads; two teams of T threads each run one packed
// two-row transform (the same code and barriers side by side) and write
// their spectrum Z back into their exchange buffer after the barrier that
// follows the step-B reads; then the CTA writes the four rows' half spectra
// as one 32-byte sector per kx (two threads per sector) instead of two half
// sectors from two CTAs (c2 row pass 3.33 -> 3.09 ms per movie).  The last
// CTA of an odd pair count runs its second team on a copy of the first pair
// and stores only the first.
template <int N1, int N2, typename Px, bool PAIRED>
__global__ void __launch_bounds__(2 * TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS / 2) k_fwd_rows2l_raw4(FwdRowsArgs a) {
  using TL = TwoLevel<N1, N2>;
  constexpr int N = TL::N, T = TL::T;
  constexpr int RB = raw_row_bytes<Px>(N);
  extern __shared__ float2 dynraw[];
  const int tid = threadIdx.x, team = tid / T, lt = tid - team * T;
  float2* ysm = dynraw + (size_t)team * N;
  unsigned char* rawb = reinterpret_cast<unsigned char*>(dynraw + 2 * N);  // four staged rows
  const int y0 = 4 * blockIdx.x;
  const bool two = y0 + 2 < a.nu;  // the second row pair exists
  const Px* f = reinterpret_cast<const Px*>(fwd_frame(a));
  auto row = [&](int j) { return f + (long long)(a.offy + y0 + (two ? j : (j & 1))) * a.nx + a.offx; };
#pragma unroll
  for (int j = 0; j < 4; j++) stage_raw_row<Px>(rawb + j * RB, row(j), N, tid, 2 * T);
  __syncthreads();
  const Px* p0 = reinterpret_cast<const Px*>(rawb + (2 * team) * RB + (reinterpret_cast<uintptr_t>(row(2 * team)) & 15));
  const Px* p1 =
      reinterpret_cast<const Px*>(rawb + (2 * team + 1) * RB + (reinterpret_cast<uintptr_t>(row(2 * team + 1)) & 15));
  TL::template run<false, true, PAIRED>(
      ysm, a.tw, [&](int x) { return make_float2((float)p0[x], (float)p1[x]); },
      [&](int k, float2 v) { ysm[k] = v; }, (N1 - 1) / 2, lt);
  __syncthreads();
  const int nh = two ? 2 : 1;
  for (int i = tid; i < 2 * a.hk; i += 2 * T) {
    const int k = i >> 1, h = i & 1;
    if (h < nh) {
      const float2* zs = dynraw + (size_t)h * N;
      const float2 z = zs[k];
      const float2 zc = zs[k == 0 ? 0 : N - k];
      const float2 X = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
      const float2 Y = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
      *reinterpret_cast<float4*>(a.outA + (long long)k * a.ldt + y0 + 2 * h) = make_float4(X.x, X.y, Y.x, Y.y);
    }
  }
}

// Forward rows: two image rows (or the two reference sets of one row) packed
// as one complex transform, then split into the two real half spectra.
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
    case MC_MODE_U8: stage_rows<uint8_t>(xin, a, r0, r1, N, TL::T); break;
    case 1: stage_rows<int16_t>(xin, a, r0, r1, N, TL::T); break;
    case 6: stage_rows<uint16_t>(xin, a, r0, r1, N, TL::T); break;
    case MC_MODE_F16: stage_rows<__half>(xin, a, r0, r1, N, TL::T); break;
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

template <int A, int B, typename PX, bool PR>
cudaError_t launch_raw_rows_p(const FwdRowsArgs& a, int grid, cudaStream_t st) {
  const size_t smem = 2 * (size_t)A * B * sizeof(float2) + 4 * (size_t)raw_row_bytes<PX>(A * B);
  cudaError_t e = allow_smem((const void*)k_fwd_rows2l_raw4<A, B, PX, PR>, smem);
  if (e != cudaSuccess) return e;
  k_fwd_rows2l_raw4<A, B, PX, PR><<<(grid + 1) / 2, 2 * TwoLevel<A, B>::T, smem, st>>>(a);
  return cudaGetLastError();
}

// Raw-row launch with the radix-53 pairing the schedule asks for (other
// lengths have no radix-53 step: one instantiation)
template <int A, int B, typename PX>
cudaError_t launch_raw_rows(const FwdRowsArgs& a, bool paired, int grid, cudaStream_t st) {
  if constexpr (A == 53) {
    if (paired != kFwdRowsPaired) return launch_raw_rows_p<A, B, PX, !kFwdRowsPaired>(a, grid, st);
  }
  return launch_raw_rows_p<A, B, PX, kFwdRowsPaired>(a, grid, st);
}

cudaError_t launch_fwd_rows2l(const FwdRowsArgs& a, cudaStream_t st) {
  int n1 = 0, n2 = 0;
  if (!two_level_split(a.nu, n1, n2)) return cudaErrorInvalidValue;
  const int grid = a.two_outputs ? a.nu : a.nu / 2;
  const bool raw = !a.two_outputs && !a.dark && !a.dark2 && !a.norm && !a.norm2;
  // the pairing of the radix-53 step (only N1 = 53 has one): schedule or built-in
  const bool paired = a.paired == 0 ? kFwdRowsPaired : a.paired == 2;
#define MC_TL_RAW(A, B, PX) return launch_raw_rows<A, B, PX>(a, paired, grid, st);
#define MC_TL_LAUNCH(A, B)                                                                           \
  if (n1 == (A) && n2 == (B)) {                                                                      \
    if (raw) {                                                                                       \
      switch (a.mode) {                                                                              \
        case 0: MC_TL_RAW(A, B, int8_t)                                                              \
        case MC_MODE_U8: MC_TL_RAW(A, B, uint8_t)                                                    \
        case 1: MC_TL_RAW(A, B, int16_t)                                                             \
        case 6: MC_TL_RAW(A, B, uint16_t)                                                            \
        case MC_MODE_F16: MC_TL_RAW(A, B, __half)                                                    \
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

}  // namespace mc
