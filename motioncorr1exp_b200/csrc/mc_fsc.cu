// FSC of -fsc (CDFAlign::PlotFSC, DFAlign.cu:212-326): the summed frames
// split into even and odd positions (raw: DFAlign.cu:806-812; corrected:
// DFAlign.cu:1142-1179, 1237-1244), per Fourier shell the cross term and the
// two powers, separately for frequencies along the drift (|cos| > cos 45°)
// and across it.  One CTA per kx column reads every summed frame's column
// once, keeps the four sums of a 2048-row chunk in shared memory, then each
// thread bins a contiguous run of rows (shell ids change rarely along a run)
// into the CTA's FP64 shell table; a second kernel adds the per-column tables
// in a fixed order.
#include "kcommon.cuh"

namespace mc {
namespace {

constexpr int kFscChunk = 2048;

__global__ void __launch_bounds__(kThreads) k_fsc_cols(FscArgs a, const float2* __restrict__ ey) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const int nh = 12 * a.nbox;
  double* hist = reinterpret_cast<double*>(fsm);               // [class][box][6]
  float2* acc = reinterpret_cast<float2*>(hist + nh);          // raw even, raw odd, corr even, corr odd
  float2* ex = acc + 4 * kFscChunk;                            // exp(+2 pi i sx kx / n) per frame
  const int tid = threadIdx.x, kx = blockIdx.x, n = a.n;
  for (int i = tid; i < nh; i += kThreads) hist[i] = 0.0;
  for (int f = tid; f < a.nsum; f += kThreads) {
    double sn, cn;
    const double t = a.shifts[f].x * (double)kx / (double)n;
    sincospi(2.0 * (t - rint(t)), &sn, &cn);
    ex[f] = make_float2((float)cn, (float)sn);
  }
  const float nsamc = (float)(n / 2 + 1);
  const float step = (float)a.step;
  for (int c0 = 0; c0 < n; c0 += kFscChunk) {
    const int len = min(kFscChunk, n - c0);
    __syncthreads();  // ex and hist ready; the previous chunk's binning is done with acc
    for (int i = tid; i < len; i += kThreads)
#pragma unroll
      for (int s = 0; s < 4; s++) acc[s * kFscChunk + i] = make_float2(0.f, 0.f);
    // each thread accumulates exactly the rows it zeroed: no barrier needed
    for (int f = 0; f < a.nsum; f++) {
      const float2* col = a.spec + (long long)a.frames[f] * a.stride + (long long)kx * a.ldn + c0;
      const float2* eyf = ey + (long long)f * n + c0;
      const float2 e = ex[f];
      const bool ap = a.apply[f] != 0;
      float2* ar = acc + (f & 1) * kFscChunk;
      float2* ac = acc + (2 + (f & 1)) * kFscChunk;
      for (int i = tid; i < len; i += kThreads) {
        const float2 v = __ldg(col + i);
        ar[i] = cadd(ar[i], v);
        ac[i] = cadd(ac[i], ap ? cmul(v, cmul(e, __ldg(eyf + i))) : v);
      }
    }
    __syncthreads();
    const int per = (len + kThreads - 1) / kThreads;
    const int i0 = min(len, tid * per), i1 = min(len, i0 + per);
    int key = -1;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int i = i0; i < i1; i++) {
      const int ky = c0 + i;
      const int y = ky < n / 2 ? ky : ky - n;  // MkPosList rows (cufunc.cu:309-339)
      const float r = sqrtf((float)(kx * kx + y * y));
      if ((int)r <= 0 || r >= nsamc) continue;
      const int id = (int)(r / step);
      // products and sum rounded separately (no FMA contraction), as the host computes them
      const double dot = __dadd_rn(__dmul_rn((double)kx, a.dirx), __dmul_rn((double)y, a.diry));
      const float angle = (float)(fabs(dot) / (double)r);
      const int k = (angle > a.edge ? 0 : a.nbox) + id;
      if (k != key) {
        if (key >= 0)
#pragma unroll
          for (int q = 0; q < 6; q++) atomicAdd(hist + key * 6 + q, s[q]);
        key = k;
#pragma unroll
        for (int q = 0; q < 6; q++) s[q] = 0.0;
      }
      const float2 r0 = acc[i], r1 = acc[kFscChunk + i], c0v = acc[2 * kFscChunk + i],
                   c1v = acc[3 * kFscChunk + i];
      s[0] += (double)r0.x * r1.x + (double)r0.y * r1.y;
      s[1] += (double)r0.x * r0.x + (double)r0.y * r0.y;
      s[2] += (double)r1.x * r1.x + (double)r1.y * r1.y;
      s[3] += (double)c0v.x * c1v.x + (double)c0v.y * c1v.y;
      s[4] += (double)c0v.x * c0v.x + (double)c0v.y * c0v.y;
      s[5] += (double)c1v.x * c1v.x + (double)c1v.y * c1v.y;
    }
    if (key >= 0)
#pragma unroll
      for (int q = 0; q < 6; q++) atomicAdd(hist + key * 6 + q, s[q]);
  }
  __syncthreads();
  double* part = a.part + (long long)kx * nh;
  for (int i = tid; i < nh; i += kThreads) part[i] = hist[i];
}

__global__ void k_fsc_reduce(const double* __restrict__ part, int H, int nh, double* out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nh; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int kx = 0; kx < H; kx++) s += part[(long long)kx * nh + e];
    out[e] = s;
  }
}

}  // namespace

size_t fsc_smem(int nbox, int nsum) {
  return sizeof(double) * 12 * (size_t)nbox + sizeof(float2) * (4 * (size_t)kFscChunk + (size_t)nsum);
}

cudaError_t launch_fsc(const FscArgs& a, float2* ey, cudaStream_t st) {
  cudaError_t e = launch_ramp(a.shifts, a.nsum, a.n, ey, st);
  if (e != cudaSuccess) return e;
  const size_t smem = fsc_smem(a.nbox, a.nsum);
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  e = allow_smem((const void*)k_fsc_cols, smem);
  if (e != cudaSuccess) return e;
  k_fsc_cols<<<a.H, kThreads, smem, st>>>(a, ey);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int nh = 12 * a.nbox;
  k_fsc_reduce<<<(nh + 255) / 256, 256, 0, st>>>(a.part, a.H, nh, a.out);
  return cudaGetLastError();
}

}  // namespace mc
