// Forward transforms of libmc (sm_100a): decode + dark/gain + crop + row FFT
// with transposed store (DFAlign.cu:710-806, general form), the column FFT with
// Fourier-crop binning (cufunc.cu:162-176, 223-227) and the batched row
// transforms of the inverse passes.  The two-level row kernels live in
// mc_fwd_raw.cu, the radix-2 split forms for lengths 2N in mc_fwd_dif.cu.
#include <algorithm>

#include "kcommon.cuh"

namespace mc {

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

// Batched rows: out_row[i] = scale * X[i < keep_lo ? i : i + (n - n_out)].
template <int N1, int N2, bool INV, bool PAIRED, bool PLAIN = false>
__global__ void __launch_bounds__(TwoLevel<N1, N2>::T, MC_TL_MIN_BLOCKS) k_rows_fft2l(RowsFftArgs a) {
  using TL = TwoLevel<N1, N2>;
  __shared__ float2 ysm[TL::N];
  const long long row = blockIdx.x;
  const float2* in = a.in + row * a.ld_in;
  float2* out = a.out + row * a.ld_out;
  if constexpr (PLAIN) {
    // every output kept, unscaled (the forward column pass without a Fourier
    // crop): no per-output crop test or multiply (2.47 -> 2.15 ms per c2 movie)
    TL::template run<INV, false, PAIRED>(ysm, a.tw, [&](int i) { return __ldg(in + i); },
                                         [&](int k, float2 v) { out[k] = v; });
  } else {
    const int shift = TL::N - a.n_out, keep = a.keep_lo;
    const float sc = a.scale;
    TL::template run<INV, false, PAIRED>(ysm, a.tw, [&](int i) { return __ldg(in + i); },
                          [&](int k, float2 v) {
                            int o;
                            if (k < keep) o = k;
                            else if (k >= keep + shift) o = k - shift;
                            else return;
                            out[o] = make_float2(v.x * sc, v.y * sc);
                          });
  }
}


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

// Forward column launch with the radix-53 pairing the schedule asks for
template <int A, int B>
void launch_cols_fwd(const RowsFftArgs& a, bool paired, cudaStream_t st) {
  const bool plain = a.n_out == A * B && a.keep_lo >= A * B && a.scale == 1.f;
  if constexpr (A == 53) {
    if (paired != kFwdColsPaired) {
      if (plain) k_rows_fft2l<A, B, false, !kFwdColsPaired, true><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a);
      else k_rows_fft2l<A, B, false, !kFwdColsPaired><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a);
      return;
    }
  }
  if (plain) k_rows_fft2l<A, B, false, kFwdColsPaired, true><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a);
  else k_rows_fft2l<A, B, false, kFwdColsPaired><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a);
}

cudaError_t launch_rows_fft2l(const RowsFftArgs& a, bool inverse, cudaStream_t st) {
  int n1 = 0, n2 = 0;
  if (!two_level_split(a.plan.n, n1, n2)) return cudaErrorInvalidValue;
  // the pairing of the radix-53 step (only N1 = 53 has one): schedule or built-in
  const bool paired = a.paired == 0 ? kFwdColsPaired : a.paired == 2;
#define MC_TL_LAUNCH(A, B)                                                                   \
  if (n1 == (A) && n2 == (B)) {                                                              \
    if (inverse) k_rows_fft2l<A, B, true, kFwdColsPaired><<<a.nrows, TwoLevel<A, B>::T, 0, st>>>(a); \
    else launch_cols_fwd<A, B>(a, paired, st);                                               \
    return cudaGetLastError();                                                               \
  }
  MC_TWO_LEVEL_LIST(MC_TL_LAUNCH)
#undef MC_TL_LAUNCH
  return cudaErrorInvalidValue;
}

}  // namespace mc
