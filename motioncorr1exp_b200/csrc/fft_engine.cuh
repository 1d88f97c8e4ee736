// Mixed-radix Stockham FFT over shared memory.
//
// A transform of length n runs as a list of stages with radices R_0..R_{s-1}
// (product n).  Stage s with span Ns = R_0*..*R_{s-1} does, for every
// butterfly j in [0, n/R):
//     v[r]  = src[j + r*n/R] * W_n^(r * (j mod Ns) * n/(Ns*R))      (r >= 1)
//     v     = DFT_R(v)
//     dst[(j div Ns)*Ns*R + (j mod Ns) + r*Ns] = v[r]
// which leaves the result in natural order (autosort) after the last stage.
// W_n = exp(-2 pi i / n) for the forward transform, its conjugate for the
// inverse; both transforms are un-normalised (cuFFT / FFTW convention).
//
// A batch of B transforms shares the stages.  Two element layouts exist:
//   rows        element (b, i) at b*ld + i   (thread index: i fastest)
//   interleaved element (b, i) at b + B*i    (thread index: b fastest)
// Both keep consecutive threads on consecutive shared-memory words.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "f2ops.cuh"
#include "dft_gen.cuh"

namespace mc {

constexpr int kMaxStages = 14;

// q = x / d, r = x % d for x < 2^22 using a float reciprocal plus one fix-up.
struct FastDiv {
  uint32_t d;
  float inv;
};

__host__ __device__ inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  f.d = d;
  f.inv = 1.0f / (float)d;
  return f;
}

__device__ __forceinline__ void fdivmod(uint32_t x, FastDiv f, uint32_t& q, uint32_t& r) {
  uint32_t qq = (uint32_t)((float)x * f.inv);
  int rr = (int)x - (int)(qq * f.d);
  if (rr < 0) {
    qq -= 1;
    rr += (int)f.d;
  } else if (rr >= (int)f.d) {
    qq += 1;
    rr -= (int)f.d;
  }
  q = qq;
  r = (uint32_t)rr;
}

struct FftStage {
  int R;          // radix
  int Ns;         // span before this stage
  int tws;        // twiddle index step n/(Ns*R)
  FastDiv nsdiv;  // divide by Ns
  FastDiv nqdiv;  // divide by n/R
};

struct FftPlan1D {
  int n;
  int nst;
  FftStage st[kMaxStages];
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// -i*z (forward) or +i*z (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 z) {
  return INV ? make_float2(-z.y, z.x) : make_float2(z.y, -z.x);
}

template <bool INV>
__device__ __forceinline__ void dft_r2(float2* v) {
  float2 a = v[0], b = v[1];
  v[0] = padd(a, b);
  v[1] = psub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft_r4(float2* v) {
  float2 t0 = padd(v[0], v[2]), t1 = psub(v[0], v[2]);
  float2 t2 = padd(v[1], v[3]), t3 = rot90<INV>(psub(v[1], v[3]));
  v[0] = padd(t0, t2);
  v[2] = psub(t0, t2);
  v[1] = padd(t1, t3);
  v[3] = psub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft_r8(float2* v) {
  const float h = 0.70710678118654752f;
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  dft_r4<INV>(e);
  dft_r4<INV>(o);
  // o[k] *= W8^k
  o[1] = INV ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
             : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
  o[2] = rot90<INV>(o[2]);
  o[3] = INV ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
             : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] = padd(e[k], o[k]);
    v[k + 4] = psub(e[k], o[k]);
  }
}

template <int R, bool INV>
__device__ __forceinline__ void dft_any(float2* v) {
  if constexpr (R == 2) dft_r2<INV>(v);
  else if constexpr (R == 4) dft_r4<INV>(v);
  else if constexpr (R == 8) dft_r8<INV>(v);
  else if constexpr (R == 3) dft_r3<INV>(v);
  else if constexpr (R == 5) dft_r5<INV>(v);
  else if constexpr (R == 7) dft_r7<INV>(v);
  else if constexpr (R == 11) dft_r11<INV>(v);
  else if constexpr (R == 13) dft_r13<INV>(v);
  else if constexpr (R == 53) dft_r53<INV>(v);
}

// One Stockham stage with compile-time radix R over B transforms.
// INTERLEAVED=false: element (b, i) at b*ld + i.  true: at b + B*i.
template <int R, bool INV, bool INTERLEAVED>
__device__ __forceinline__ void stage_fixed(const float2* __restrict__ src, float2* __restrict__ dst,
                                            const FftStage& s, int B, FastDiv bdiv, int ld,
                                            const float2* __restrict__ tw, int tid, int nth) {
  const int nq = (int)s.nqdiv.d;
  const int total = nq * B;
  for (int t = tid; t < total; t += nth) {
    uint32_t j, b;
    if (INTERLEAVED) fdivmod((uint32_t)t, bdiv, j, b);
    else fdivmod((uint32_t)t, s.nqdiv, b, j);
    uint32_t jq, jm;
    fdivmod(j, s.nsdiv, jq, jm);
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = (int)j + r * nq;
      v[r] = INTERLEAVED ? src[b + B * i] : src[b * ld + i];
    }
    if (s.Ns > 1) {
      const int step = (int)jm * s.tws;
#pragma unroll
      for (int r = 1; r < R; r++) {
        float2 w = tw[r * step];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dft_any<R, INV>(v);
    const int base = (int)jq * s.Ns * R + (int)jm;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = base + r * s.Ns;
      if (INTERLEAVED) dst[b + B * i] = v[r];
      else dst[b * ld + i] = v[r];
    }
  }
}

// Radix-53 stage with every butterfly spread over kSplit53 threads: each
// thread loads the 53 inputs and produces its share of the outputs.  The
// stage has only n/53 butterflies per transform, so this keeps the CTA busy.
template <bool INV, bool INTERLEAVED>
__device__ __forceinline__ void stage_r53_split(const float2* __restrict__ src, float2* __restrict__ dst,
                                                const FftStage& s, int B, FastDiv bdiv, int ld,
                                                const float2* __restrict__ tw, int tid, int nth) {
  constexpr int R = 53;
  const int nq = (int)s.nqdiv.d;
  const int total = nq * B * kSplit53;
  const FastDiv sdiv = make_fastdiv((uint32_t)kSplit53);
  for (int t = tid; t < total; t += nth) {
    uint32_t jb, part;
    fdivmod((uint32_t)t, sdiv, jb, part);
    uint32_t j, b;
    if (INTERLEAVED) fdivmod(jb, bdiv, j, b);
    else fdivmod(jb, s.nqdiv, b, j);
    uint32_t jq, jm;
    fdivmod(j, s.nsdiv, jq, jm);
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = (int)j + r * nq;
      v[r] = INTERLEAVED ? src[b + B * i] : src[b * ld + i];
    }
    if (s.Ns > 1) {
      const int step = (int)jm * s.tws;
#pragma unroll
      for (int r = 1; r < R; r++) {
        float2 w = tw[r * step];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    const int base = (int)jq * s.Ns * R + (int)jm;
    dft_r53_part<INV>(v, (int)part, [&](int r, float2 x) {
      const int i = base + r * s.Ns;
      if (INTERLEAVED) dst[b + B * i] = x;
      else dst[b * ld + i] = x;
    });
  }
}

// Runtime-radix fallback: every output of every butterfly as a direct sum,
//   X_k = sum_r src[j + r*n/R] * W_n^(r*((j mod Ns)*tws + k*n/R)).
template <bool INV, bool INTERLEAVED>
__device__ void stage_generic(const float2* __restrict__ src, float2* __restrict__ dst, const FftStage& s,
                              int n, int B, FastDiv bdiv, int ld, const float2* __restrict__ tw, int tid,
                              int nth) {
  const int R = s.R;
  const int nq = (int)s.nqdiv.d;
  const int total = nq * B * R;
  const FastDiv rdiv = make_fastdiv((uint32_t)R);
  for (int t = tid; t < total; t += nth) {
    uint32_t jb, k;
    fdivmod((uint32_t)t, rdiv, jb, k);
    uint32_t j, b;
    if (INTERLEAVED) fdivmod(jb, bdiv, j, b);
    else fdivmod(jb, s.nqdiv, b, j);
    uint32_t jq, jm;
    fdivmod(j, s.nsdiv, jq, jm);
    const int step = ((int)jm * s.tws + (int)k * nq) % n;
    int e = 0;
    float2 acc = make_float2(0.f, 0.f);
    for (int r = 0; r < R; r++) {
      const int i = (int)j + r * nq;
      const float2 x = INTERLEAVED ? src[b + B * i] : src[b * ld + i];
      float2 w = tw[e];
      if (INV) w.y = -w.y;
      const float2 p = cmul(x, w);
      acc.x += p.x;
      acc.y += p.y;
      e += step;
      if (e >= n) e -= n;
    }
    const int i = (int)jq * s.Ns * R + (int)jm + (int)k * s.Ns;
    if (INTERLEAVED) dst[b + B * i] = acc;
    else dst[b * ld + i] = acc;
  }
}

// Runs all stages; a and b are the two shared-memory buffers.  Returns the
// buffer holding the result.  Ends with a __syncthreads().
template <bool INV, bool INTERLEAVED>
__device__ float2* fft_run(float2* a, float2* b, const FftPlan1D& p, int B, int ld,
                           const float2* __restrict__ tw, int tid, int nth) {
  const FastDiv bdiv = make_fastdiv((uint32_t)B);
  for (int si = 0; si < p.nst; si++) {
    const FftStage& s = p.st[si];
    switch (s.R) {
      case 2: stage_fixed<2, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 3: stage_fixed<3, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 4: stage_fixed<4, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 5: stage_fixed<5, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 7: stage_fixed<7, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 8: stage_fixed<8, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 11: stage_fixed<11, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 13: stage_fixed<13, INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      case 53: stage_r53_split<INV, INTERLEAVED>(a, b, s, B, bdiv, ld, tw, tid, nth); break;
      default: stage_generic<INV, INTERLEAVED>(a, b, s, p.n, B, bdiv, ld, tw, tid, nth); break;
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
  }
  return a;
}

}  // namespace mc
