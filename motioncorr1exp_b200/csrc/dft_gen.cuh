// Generated by gen_dft.py -- do not edit by hand.
// Straight-line odd-radix DFT butterflies (symmetric direct form).
#pragma once
#include <cuda_runtime.h>
#include "f2ops.cuh"
// MC_PACKED_FMA=1: the odd butterflies' sums on packed FP32 pairs (bitwise
// the same results: each half is the scalar FMA chain)
#ifndef MC_PACKED_FMA
#define MC_PACKED_FMA 0
#endif
namespace mc {
constexpr int kGeneratedOddRadices[] = {3, 5, 7, 11, 13, 53};
template <bool INV> __device__ __forceinline__ void dft_r3(float2* v) {
  const float2 x0 = v[0];
#if MC_PACKED_FMA
  const f2reg S1 = f2pk(padd(v[1], v[2]));
  const f2reg D1 = f2pk(psub(v[1], v[2]));
  { float2 t = f2up(S1);
    v[0] = make_float2(x0.x + t.x, x0.y + t.y); }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.5f), A); B = f2fma(D1, f2splat(0.8660253882408142f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[1] = make_float2(a.x + b.y, a.y - b.x); v[2] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[1] = make_float2(a.x - b.y, a.y + b.x); v[2] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
#else
  const float2 s1 = padd(v[1], v[2]);
  const float2 d1 = psub(v[1], v[2]);
  v[0] = make_float2(x0.x + (s1.x), x0.y + (s1.y));
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.5f, ar); ai = fmaf(s1.y, -0.5f, ai); br = fmaf(d1.x, 0.8660253882408142f, br); bi = fmaf(d1.y, 0.8660253882408142f, bi);
    if (!INV) {
      v[1] = make_float2(ar + bi, ai - br); v[2] = make_float2(ar - bi, ai + br);
    } else {
      v[1] = make_float2(ar - bi, ai + br); v[2] = make_float2(ar + bi, ai - br);
    }
  }
#endif
}
template <bool INV> __device__ __forceinline__ void dft_r5(float2* v) {
  const float2 x0 = v[0];
#if MC_PACKED_FMA
  const f2reg S1 = f2pk(padd(v[1], v[4]));
  const f2reg D1 = f2pk(psub(v[1], v[4]));
  const f2reg S2 = f2pk(padd(v[2], v[3]));
  const f2reg D2 = f2pk(psub(v[2], v[3]));
  { float2 t = f2up(S1);
    { const float2 u = f2up(S2); t.x += u.x; t.y += u.y; }
    v[0] = make_float2(x0.x + t.x, x0.y + t.y); }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(0.30901700258255005f), A); B = f2fma(D1, f2splat(0.9510565400123596f), B);
    A = f2fma(S2, f2splat(-0.80901700258255f), A); B = f2fma(D2, f2splat(0.5877852439880371f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[1] = make_float2(a.x + b.y, a.y - b.x); v[4] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[1] = make_float2(a.x - b.y, a.y + b.x); v[4] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.80901700258255f), A); B = f2fma(D1, f2splat(0.5877852439880371f), B);
    A = f2fma(S2, f2splat(0.30901700258255005f), A); B = f2fma(D2, f2splat(-0.9510565400123596f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[2] = make_float2(a.x + b.y, a.y - b.x); v[3] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[2] = make_float2(a.x - b.y, a.y + b.x); v[3] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
#else
  const float2 s1 = padd(v[1], v[4]);
  const float2 d1 = psub(v[1], v[4]);
  const float2 s2 = padd(v[2], v[3]);
  const float2 d2 = psub(v[2], v[3]);
  v[0] = make_float2(x0.x + (s1.x + s2.x), x0.y + (s1.y + s2.y));
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.30901700258255005f, ar); ai = fmaf(s1.y, 0.30901700258255005f, ai); br = fmaf(d1.x, 0.9510565400123596f, br); bi = fmaf(d1.y, 0.9510565400123596f, bi);
    ar = fmaf(s2.x, -0.80901700258255f, ar); ai = fmaf(s2.y, -0.80901700258255f, ai); br = fmaf(d2.x, 0.5877852439880371f, br); bi = fmaf(d2.y, 0.5877852439880371f, bi);
    if (!INV) {
      v[1] = make_float2(ar + bi, ai - br); v[4] = make_float2(ar - bi, ai + br);
    } else {
      v[1] = make_float2(ar - bi, ai + br); v[4] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.80901700258255f, ar); ai = fmaf(s1.y, -0.80901700258255f, ai); br = fmaf(d1.x, 0.5877852439880371f, br); bi = fmaf(d1.y, 0.5877852439880371f, bi);
    ar = fmaf(s2.x, 0.30901700258255005f, ar); ai = fmaf(s2.y, 0.30901700258255005f, ai); br = fmaf(d2.x, -0.9510565400123596f, br); bi = fmaf(d2.y, -0.9510565400123596f, bi);
    if (!INV) {
      v[2] = make_float2(ar + bi, ai - br); v[3] = make_float2(ar - bi, ai + br);
    } else {
      v[2] = make_float2(ar - bi, ai + br); v[3] = make_float2(ar + bi, ai - br);
    }
  }
#endif
}
template <bool INV> __device__ __forceinline__ void dft_r7(float2* v) {
  const float2 x0 = v[0];
#if MC_PACKED_FMA
  const f2reg S1 = f2pk(padd(v[1], v[6]));
  const f2reg D1 = f2pk(psub(v[1], v[6]));
  const f2reg S2 = f2pk(padd(v[2], v[5]));
  const f2reg D2 = f2pk(psub(v[2], v[5]));
  const f2reg S3 = f2pk(padd(v[3], v[4]));
  const f2reg D3 = f2pk(psub(v[3], v[4]));
  { float2 t = f2up(S1);
    { const float2 u = f2up(S2); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S3); t.x += u.x; t.y += u.y; }
    v[0] = make_float2(x0.x + t.x, x0.y + t.y); }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(0.6234897971153259f), A); B = f2fma(D1, f2splat(0.7818315029144287f), B);
    A = f2fma(S2, f2splat(-0.22252093255519867f), A); B = f2fma(D2, f2splat(0.9749279022216797f), B);
    A = f2fma(S3, f2splat(-0.9009688496589661f), A); B = f2fma(D3, f2splat(0.4338837265968323f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[1] = make_float2(a.x + b.y, a.y - b.x); v[6] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[1] = make_float2(a.x - b.y, a.y + b.x); v[6] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.22252093255519867f), A); B = f2fma(D1, f2splat(0.9749279022216797f), B);
    A = f2fma(S2, f2splat(-0.9009688496589661f), A); B = f2fma(D2, f2splat(-0.4338837265968323f), B);
    A = f2fma(S3, f2splat(0.6234897971153259f), A); B = f2fma(D3, f2splat(-0.7818315029144287f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[2] = make_float2(a.x + b.y, a.y - b.x); v[5] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[2] = make_float2(a.x - b.y, a.y + b.x); v[5] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.9009688496589661f), A); B = f2fma(D1, f2splat(0.4338837265968323f), B);
    A = f2fma(S2, f2splat(0.6234897971153259f), A); B = f2fma(D2, f2splat(-0.7818315029144287f), B);
    A = f2fma(S3, f2splat(-0.22252093255519867f), A); B = f2fma(D3, f2splat(0.9749279022216797f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[3] = make_float2(a.x + b.y, a.y - b.x); v[4] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[3] = make_float2(a.x - b.y, a.y + b.x); v[4] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
#else
  const float2 s1 = padd(v[1], v[6]);
  const float2 d1 = psub(v[1], v[6]);
  const float2 s2 = padd(v[2], v[5]);
  const float2 d2 = psub(v[2], v[5]);
  const float2 s3 = padd(v[3], v[4]);
  const float2 d3 = psub(v[3], v[4]);
  v[0] = make_float2(x0.x + (s1.x + s2.x + s3.x), x0.y + (s1.y + s2.y + s3.y));
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.6234897971153259f, ar); ai = fmaf(s1.y, 0.6234897971153259f, ai); br = fmaf(d1.x, 0.7818315029144287f, br); bi = fmaf(d1.y, 0.7818315029144287f, bi);
    ar = fmaf(s2.x, -0.22252093255519867f, ar); ai = fmaf(s2.y, -0.22252093255519867f, ai); br = fmaf(d2.x, 0.9749279022216797f, br); bi = fmaf(d2.y, 0.9749279022216797f, bi);
    ar = fmaf(s3.x, -0.9009688496589661f, ar); ai = fmaf(s3.y, -0.9009688496589661f, ai); br = fmaf(d3.x, 0.4338837265968323f, br); bi = fmaf(d3.y, 0.4338837265968323f, bi);
    if (!INV) {
      v[1] = make_float2(ar + bi, ai - br); v[6] = make_float2(ar - bi, ai + br);
    } else {
      v[1] = make_float2(ar - bi, ai + br); v[6] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.22252093255519867f, ar); ai = fmaf(s1.y, -0.22252093255519867f, ai); br = fmaf(d1.x, 0.9749279022216797f, br); bi = fmaf(d1.y, 0.9749279022216797f, bi);
    ar = fmaf(s2.x, -0.9009688496589661f, ar); ai = fmaf(s2.y, -0.9009688496589661f, ai); br = fmaf(d2.x, -0.4338837265968323f, br); bi = fmaf(d2.y, -0.4338837265968323f, bi);
    ar = fmaf(s3.x, 0.6234897971153259f, ar); ai = fmaf(s3.y, 0.6234897971153259f, ai); br = fmaf(d3.x, -0.7818315029144287f, br); bi = fmaf(d3.y, -0.7818315029144287f, bi);
    if (!INV) {
      v[2] = make_float2(ar + bi, ai - br); v[5] = make_float2(ar - bi, ai + br);
    } else {
      v[2] = make_float2(ar - bi, ai + br); v[5] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.9009688496589661f, ar); ai = fmaf(s1.y, -0.9009688496589661f, ai); br = fmaf(d1.x, 0.4338837265968323f, br); bi = fmaf(d1.y, 0.4338837265968323f, bi);
    ar = fmaf(s2.x, 0.6234897971153259f, ar); ai = fmaf(s2.y, 0.6234897971153259f, ai); br = fmaf(d2.x, -0.7818315029144287f, br); bi = fmaf(d2.y, -0.7818315029144287f, bi);
    ar = fmaf(s3.x, -0.22252093255519867f, ar); ai = fmaf(s3.y, -0.22252093255519867f, ai); br = fmaf(d3.x, 0.9749279022216797f, br); bi = fmaf(d3.y, 0.9749279022216797f, bi);
    if (!INV) {
      v[3] = make_float2(ar + bi, ai - br); v[4] = make_float2(ar - bi, ai + br);
    } else {
      v[3] = make_float2(ar - bi, ai + br); v[4] = make_float2(ar + bi, ai - br);
    }
  }
#endif
}
template <bool INV> __device__ __forceinline__ void dft_r11(float2* v) {
  const float2 x0 = v[0];
#if MC_PACKED_FMA
  const f2reg S1 = f2pk(padd(v[1], v[10]));
  const f2reg D1 = f2pk(psub(v[1], v[10]));
  const f2reg S2 = f2pk(padd(v[2], v[9]));
  const f2reg D2 = f2pk(psub(v[2], v[9]));
  const f2reg S3 = f2pk(padd(v[3], v[8]));
  const f2reg D3 = f2pk(psub(v[3], v[8]));
  const f2reg S4 = f2pk(padd(v[4], v[7]));
  const f2reg D4 = f2pk(psub(v[4], v[7]));
  const f2reg S5 = f2pk(padd(v[5], v[6]));
  const f2reg D5 = f2pk(psub(v[5], v[6]));
  { float2 t = f2up(S1);
    { const float2 u = f2up(S2); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S3); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S4); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S5); t.x += u.x; t.y += u.y; }
    v[0] = make_float2(x0.x + t.x, x0.y + t.y); }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(0.8412535190582275f), A); B = f2fma(D1, f2splat(0.5406408309936523f), B);
    A = f2fma(S2, f2splat(0.4154150187969208f), A); B = f2fma(D2, f2splat(0.9096319675445557f), B);
    A = f2fma(S3, f2splat(-0.1423148363828659f), A); B = f2fma(D3, f2splat(0.9898214340209961f), B);
    A = f2fma(S4, f2splat(-0.6548607349395752f), A); B = f2fma(D4, f2splat(0.7557495832443237f), B);
    A = f2fma(S5, f2splat(-0.9594929814338684f), A); B = f2fma(D5, f2splat(0.28173255920410156f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[1] = make_float2(a.x + b.y, a.y - b.x); v[10] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[1] = make_float2(a.x - b.y, a.y + b.x); v[10] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(0.4154150187969208f), A); B = f2fma(D1, f2splat(0.9096319675445557f), B);
    A = f2fma(S2, f2splat(-0.6548607349395752f), A); B = f2fma(D2, f2splat(0.7557495832443237f), B);
    A = f2fma(S3, f2splat(-0.9594929814338684f), A); B = f2fma(D3, f2splat(-0.28173255920410156f), B);
    A = f2fma(S4, f2splat(-0.1423148363828659f), A); B = f2fma(D4, f2splat(-0.9898214340209961f), B);
    A = f2fma(S5, f2splat(0.8412535190582275f), A); B = f2fma(D5, f2splat(-0.5406408309936523f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[2] = make_float2(a.x + b.y, a.y - b.x); v[9] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[2] = make_float2(a.x - b.y, a.y + b.x); v[9] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.1423148363828659f), A); B = f2fma(D1, f2splat(0.9898214340209961f), B);
    A = f2fma(S2, f2splat(-0.9594929814338684f), A); B = f2fma(D2, f2splat(-0.28173255920410156f), B);
    A = f2fma(S3, f2splat(0.4154150187969208f), A); B = f2fma(D3, f2splat(-0.9096319675445557f), B);
    A = f2fma(S4, f2splat(0.8412535190582275f), A); B = f2fma(D4, f2splat(0.5406408309936523f), B);
    A = f2fma(S5, f2splat(-0.6548607349395752f), A); B = f2fma(D5, f2splat(0.7557495832443237f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[3] = make_float2(a.x + b.y, a.y - b.x); v[8] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[3] = make_float2(a.x - b.y, a.y + b.x); v[8] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.6548607349395752f), A); B = f2fma(D1, f2splat(0.7557495832443237f), B);
    A = f2fma(S2, f2splat(-0.1423148363828659f), A); B = f2fma(D2, f2splat(-0.9898214340209961f), B);
    A = f2fma(S3, f2splat(0.8412535190582275f), A); B = f2fma(D3, f2splat(0.5406408309936523f), B);
    A = f2fma(S4, f2splat(-0.9594929814338684f), A); B = f2fma(D4, f2splat(0.28173255920410156f), B);
    A = f2fma(S5, f2splat(0.4154150187969208f), A); B = f2fma(D5, f2splat(-0.9096319675445557f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[4] = make_float2(a.x + b.y, a.y - b.x); v[7] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[4] = make_float2(a.x - b.y, a.y + b.x); v[7] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.9594929814338684f), A); B = f2fma(D1, f2splat(0.28173255920410156f), B);
    A = f2fma(S2, f2splat(0.8412535190582275f), A); B = f2fma(D2, f2splat(-0.5406408309936523f), B);
    A = f2fma(S3, f2splat(-0.6548607349395752f), A); B = f2fma(D3, f2splat(0.7557495832443237f), B);
    A = f2fma(S4, f2splat(0.4154150187969208f), A); B = f2fma(D4, f2splat(-0.9096319675445557f), B);
    A = f2fma(S5, f2splat(-0.1423148363828659f), A); B = f2fma(D5, f2splat(0.9898214340209961f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[5] = make_float2(a.x + b.y, a.y - b.x); v[6] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[5] = make_float2(a.x - b.y, a.y + b.x); v[6] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
#else
  const float2 s1 = padd(v[1], v[10]);
  const float2 d1 = psub(v[1], v[10]);
  const float2 s2 = padd(v[2], v[9]);
  const float2 d2 = psub(v[2], v[9]);
  const float2 s3 = padd(v[3], v[8]);
  const float2 d3 = psub(v[3], v[8]);
  const float2 s4 = padd(v[4], v[7]);
  const float2 d4 = psub(v[4], v[7]);
  const float2 s5 = padd(v[5], v[6]);
  const float2 d5 = psub(v[5], v[6]);
  v[0] = make_float2(x0.x + (s1.x + s2.x + s3.x + s4.x + s5.x), x0.y + (s1.y + s2.y + s3.y + s4.y + s5.y));
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.8412535190582275f, ar); ai = fmaf(s1.y, 0.8412535190582275f, ai); br = fmaf(d1.x, 0.5406408309936523f, br); bi = fmaf(d1.y, 0.5406408309936523f, bi);
    ar = fmaf(s2.x, 0.4154150187969208f, ar); ai = fmaf(s2.y, 0.4154150187969208f, ai); br = fmaf(d2.x, 0.9096319675445557f, br); bi = fmaf(d2.y, 0.9096319675445557f, bi);
    ar = fmaf(s3.x, -0.1423148363828659f, ar); ai = fmaf(s3.y, -0.1423148363828659f, ai); br = fmaf(d3.x, 0.9898214340209961f, br); bi = fmaf(d3.y, 0.9898214340209961f, bi);
    ar = fmaf(s4.x, -0.6548607349395752f, ar); ai = fmaf(s4.y, -0.6548607349395752f, ai); br = fmaf(d4.x, 0.7557495832443237f, br); bi = fmaf(d4.y, 0.7557495832443237f, bi);
    ar = fmaf(s5.x, -0.9594929814338684f, ar); ai = fmaf(s5.y, -0.9594929814338684f, ai); br = fmaf(d5.x, 0.28173255920410156f, br); bi = fmaf(d5.y, 0.28173255920410156f, bi);
    if (!INV) {
      v[1] = make_float2(ar + bi, ai - br); v[10] = make_float2(ar - bi, ai + br);
    } else {
      v[1] = make_float2(ar - bi, ai + br); v[10] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.4154150187969208f, ar); ai = fmaf(s1.y, 0.4154150187969208f, ai); br = fmaf(d1.x, 0.9096319675445557f, br); bi = fmaf(d1.y, 0.9096319675445557f, bi);
    ar = fmaf(s2.x, -0.6548607349395752f, ar); ai = fmaf(s2.y, -0.6548607349395752f, ai); br = fmaf(d2.x, 0.7557495832443237f, br); bi = fmaf(d2.y, 0.7557495832443237f, bi);
    ar = fmaf(s3.x, -0.9594929814338684f, ar); ai = fmaf(s3.y, -0.9594929814338684f, ai); br = fmaf(d3.x, -0.28173255920410156f, br); bi = fmaf(d3.y, -0.28173255920410156f, bi);
    ar = fmaf(s4.x, -0.1423148363828659f, ar); ai = fmaf(s4.y, -0.1423148363828659f, ai); br = fmaf(d4.x, -0.9898214340209961f, br); bi = fmaf(d4.y, -0.9898214340209961f, bi);
    ar = fmaf(s5.x, 0.8412535190582275f, ar); ai = fmaf(s5.y, 0.8412535190582275f, ai); br = fmaf(d5.x, -0.5406408309936523f, br); bi = fmaf(d5.y, -0.5406408309936523f, bi);
    if (!INV) {
      v[2] = make_float2(ar + bi, ai - br); v[9] = make_float2(ar - bi, ai + br);
    } else {
      v[2] = make_float2(ar - bi, ai + br); v[9] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.1423148363828659f, ar); ai = fmaf(s1.y, -0.1423148363828659f, ai); br = fmaf(d1.x, 0.9898214340209961f, br); bi = fmaf(d1.y, 0.9898214340209961f, bi);
    ar = fmaf(s2.x, -0.9594929814338684f, ar); ai = fmaf(s2.y, -0.9594929814338684f, ai); br = fmaf(d2.x, -0.28173255920410156f, br); bi = fmaf(d2.y, -0.28173255920410156f, bi);
    ar = fmaf(s3.x, 0.4154150187969208f, ar); ai = fmaf(s3.y, 0.4154150187969208f, ai); br = fmaf(d3.x, -0.9096319675445557f, br); bi = fmaf(d3.y, -0.9096319675445557f, bi);
    ar = fmaf(s4.x, 0.8412535190582275f, ar); ai = fmaf(s4.y, 0.8412535190582275f, ai); br = fmaf(d4.x, 0.5406408309936523f, br); bi = fmaf(d4.y, 0.5406408309936523f, bi);
    ar = fmaf(s5.x, -0.6548607349395752f, ar); ai = fmaf(s5.y, -0.6548607349395752f, ai); br = fmaf(d5.x, 0.7557495832443237f, br); bi = fmaf(d5.y, 0.7557495832443237f, bi);
    if (!INV) {
      v[3] = make_float2(ar + bi, ai - br); v[8] = make_float2(ar - bi, ai + br);
    } else {
      v[3] = make_float2(ar - bi, ai + br); v[8] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.6548607349395752f, ar); ai = fmaf(s1.y, -0.6548607349395752f, ai); br = fmaf(d1.x, 0.7557495832443237f, br); bi = fmaf(d1.y, 0.7557495832443237f, bi);
    ar = fmaf(s2.x, -0.1423148363828659f, ar); ai = fmaf(s2.y, -0.1423148363828659f, ai); br = fmaf(d2.x, -0.9898214340209961f, br); bi = fmaf(d2.y, -0.9898214340209961f, bi);
    ar = fmaf(s3.x, 0.8412535190582275f, ar); ai = fmaf(s3.y, 0.8412535190582275f, ai); br = fmaf(d3.x, 0.5406408309936523f, br); bi = fmaf(d3.y, 0.5406408309936523f, bi);
    ar = fmaf(s4.x, -0.9594929814338684f, ar); ai = fmaf(s4.y, -0.9594929814338684f, ai); br = fmaf(d4.x, 0.28173255920410156f, br); bi = fmaf(d4.y, 0.28173255920410156f, bi);
    ar = fmaf(s5.x, 0.4154150187969208f, ar); ai = fmaf(s5.y, 0.4154150187969208f, ai); br = fmaf(d5.x, -0.9096319675445557f, br); bi = fmaf(d5.y, -0.9096319675445557f, bi);
    if (!INV) {
      v[4] = make_float2(ar + bi, ai - br); v[7] = make_float2(ar - bi, ai + br);
    } else {
      v[4] = make_float2(ar - bi, ai + br); v[7] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.9594929814338684f, ar); ai = fmaf(s1.y, -0.9594929814338684f, ai); br = fmaf(d1.x, 0.28173255920410156f, br); bi = fmaf(d1.y, 0.28173255920410156f, bi);
    ar = fmaf(s2.x, 0.8412535190582275f, ar); ai = fmaf(s2.y, 0.8412535190582275f, ai); br = fmaf(d2.x, -0.5406408309936523f, br); bi = fmaf(d2.y, -0.5406408309936523f, bi);
    ar = fmaf(s3.x, -0.6548607349395752f, ar); ai = fmaf(s3.y, -0.6548607349395752f, ai); br = fmaf(d3.x, 0.7557495832443237f, br); bi = fmaf(d3.y, 0.7557495832443237f, bi);
    ar = fmaf(s4.x, 0.4154150187969208f, ar); ai = fmaf(s4.y, 0.4154150187969208f, ai); br = fmaf(d4.x, -0.9096319675445557f, br); bi = fmaf(d4.y, -0.9096319675445557f, bi);
    ar = fmaf(s5.x, -0.1423148363828659f, ar); ai = fmaf(s5.y, -0.1423148363828659f, ai); br = fmaf(d5.x, 0.9898214340209961f, br); bi = fmaf(d5.y, 0.9898214340209961f, bi);
    if (!INV) {
      v[5] = make_float2(ar + bi, ai - br); v[6] = make_float2(ar - bi, ai + br);
    } else {
      v[5] = make_float2(ar - bi, ai + br); v[6] = make_float2(ar + bi, ai - br);
    }
  }
#endif
}
template <bool INV> __device__ __forceinline__ void dft_r13(float2* v) {
  const float2 x0 = v[0];
#if MC_PACKED_FMA
  const f2reg S1 = f2pk(padd(v[1], v[12]));
  const f2reg D1 = f2pk(psub(v[1], v[12]));
  const f2reg S2 = f2pk(padd(v[2], v[11]));
  const f2reg D2 = f2pk(psub(v[2], v[11]));
  const f2reg S3 = f2pk(padd(v[3], v[10]));
  const f2reg D3 = f2pk(psub(v[3], v[10]));
  const f2reg S4 = f2pk(padd(v[4], v[9]));
  const f2reg D4 = f2pk(psub(v[4], v[9]));
  const f2reg S5 = f2pk(padd(v[5], v[8]));
  const f2reg D5 = f2pk(psub(v[5], v[8]));
  const f2reg S6 = f2pk(padd(v[6], v[7]));
  const f2reg D6 = f2pk(psub(v[6], v[7]));
  { float2 t = f2up(S1);
    { const float2 u = f2up(S2); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S3); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S4); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S5); t.x += u.x; t.y += u.y; }
    { const float2 u = f2up(S6); t.x += u.x; t.y += u.y; }
    v[0] = make_float2(x0.x + t.x, x0.y + t.y); }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(0.8854560256004333f), A); B = f2fma(D1, f2splat(0.4647231698036194f), B);
    A = f2fma(S2, f2splat(0.5680647492408752f), A); B = f2fma(D2, f2splat(0.8229838609695435f), B);
    A = f2fma(S3, f2splat(0.1205366775393486f), A); B = f2fma(D3, f2splat(0.9927088618278503f), B);
    A = f2fma(S4, f2splat(-0.35460489988327026f), A); B = f2fma(D4, f2splat(0.9350162148475647f), B);
    A = f2fma(S5, f2splat(-0.7485107779502869f), A); B = f2fma(D5, f2splat(0.6631226539611816f), B);
    A = f2fma(S6, f2splat(-0.9709418416023254f), A); B = f2fma(D6, f2splat(0.23931565880775452f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[1] = make_float2(a.x + b.y, a.y - b.x); v[12] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[1] = make_float2(a.x - b.y, a.y + b.x); v[12] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(0.5680647492408752f), A); B = f2fma(D1, f2splat(0.8229838609695435f), B);
    A = f2fma(S2, f2splat(-0.35460489988327026f), A); B = f2fma(D2, f2splat(0.9350162148475647f), B);
    A = f2fma(S3, f2splat(-0.9709418416023254f), A); B = f2fma(D3, f2splat(0.23931565880775452f), B);
    A = f2fma(S4, f2splat(-0.7485107779502869f), A); B = f2fma(D4, f2splat(-0.6631226539611816f), B);
    A = f2fma(S5, f2splat(0.1205366775393486f), A); B = f2fma(D5, f2splat(-0.9927088618278503f), B);
    A = f2fma(S6, f2splat(0.8854560256004333f), A); B = f2fma(D6, f2splat(-0.4647231698036194f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[2] = make_float2(a.x + b.y, a.y - b.x); v[11] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[2] = make_float2(a.x - b.y, a.y + b.x); v[11] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(0.1205366775393486f), A); B = f2fma(D1, f2splat(0.9927088618278503f), B);
    A = f2fma(S2, f2splat(-0.9709418416023254f), A); B = f2fma(D2, f2splat(0.23931565880775452f), B);
    A = f2fma(S3, f2splat(-0.35460489988327026f), A); B = f2fma(D3, f2splat(-0.9350162148475647f), B);
    A = f2fma(S4, f2splat(0.8854560256004333f), A); B = f2fma(D4, f2splat(-0.4647231698036194f), B);
    A = f2fma(S5, f2splat(0.5680647492408752f), A); B = f2fma(D5, f2splat(0.8229838609695435f), B);
    A = f2fma(S6, f2splat(-0.7485107779502869f), A); B = f2fma(D6, f2splat(0.6631226539611816f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[3] = make_float2(a.x + b.y, a.y - b.x); v[10] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[3] = make_float2(a.x - b.y, a.y + b.x); v[10] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.35460489988327026f), A); B = f2fma(D1, f2splat(0.9350162148475647f), B);
    A = f2fma(S2, f2splat(-0.7485107779502869f), A); B = f2fma(D2, f2splat(-0.6631226539611816f), B);
    A = f2fma(S3, f2splat(0.8854560256004333f), A); B = f2fma(D3, f2splat(-0.4647231698036194f), B);
    A = f2fma(S4, f2splat(0.1205366775393486f), A); B = f2fma(D4, f2splat(0.9927088618278503f), B);
    A = f2fma(S5, f2splat(-0.9709418416023254f), A); B = f2fma(D5, f2splat(-0.23931565880775452f), B);
    A = f2fma(S6, f2splat(0.5680647492408752f), A); B = f2fma(D6, f2splat(-0.8229838609695435f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[4] = make_float2(a.x + b.y, a.y - b.x); v[9] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[4] = make_float2(a.x - b.y, a.y + b.x); v[9] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.7485107779502869f), A); B = f2fma(D1, f2splat(0.6631226539611816f), B);
    A = f2fma(S2, f2splat(0.1205366775393486f), A); B = f2fma(D2, f2splat(-0.9927088618278503f), B);
    A = f2fma(S3, f2splat(0.5680647492408752f), A); B = f2fma(D3, f2splat(0.8229838609695435f), B);
    A = f2fma(S4, f2splat(-0.9709418416023254f), A); B = f2fma(D4, f2splat(-0.23931565880775452f), B);
    A = f2fma(S5, f2splat(0.8854560256004333f), A); B = f2fma(D5, f2splat(-0.4647231698036194f), B);
    A = f2fma(S6, f2splat(-0.35460489988327026f), A); B = f2fma(D6, f2splat(0.9350162148475647f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[5] = make_float2(a.x + b.y, a.y - b.x); v[8] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[5] = make_float2(a.x - b.y, a.y + b.x); v[8] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
  {
    f2reg A = f2pk(x0), B = 0ull;
    A = f2fma(S1, f2splat(-0.9709418416023254f), A); B = f2fma(D1, f2splat(0.23931565880775452f), B);
    A = f2fma(S2, f2splat(0.8854560256004333f), A); B = f2fma(D2, f2splat(-0.4647231698036194f), B);
    A = f2fma(S3, f2splat(-0.7485107779502869f), A); B = f2fma(D3, f2splat(0.6631226539611816f), B);
    A = f2fma(S4, f2splat(0.5680647492408752f), A); B = f2fma(D4, f2splat(-0.8229838609695435f), B);
    A = f2fma(S5, f2splat(-0.35460489988327026f), A); B = f2fma(D5, f2splat(0.9350162148475647f), B);
    A = f2fma(S6, f2splat(0.1205366775393486f), A); B = f2fma(D6, f2splat(-0.9927088618278503f), B);
    const float2 a = f2up(A), b = f2up(B);
    if (!INV) {
      v[6] = make_float2(a.x + b.y, a.y - b.x); v[7] = make_float2(a.x - b.y, a.y + b.x);
    } else {
      v[6] = make_float2(a.x - b.y, a.y + b.x); v[7] = make_float2(a.x + b.y, a.y - b.x);
    }
  }
#else
  const float2 s1 = padd(v[1], v[12]);
  const float2 d1 = psub(v[1], v[12]);
  const float2 s2 = padd(v[2], v[11]);
  const float2 d2 = psub(v[2], v[11]);
  const float2 s3 = padd(v[3], v[10]);
  const float2 d3 = psub(v[3], v[10]);
  const float2 s4 = padd(v[4], v[9]);
  const float2 d4 = psub(v[4], v[9]);
  const float2 s5 = padd(v[5], v[8]);
  const float2 d5 = psub(v[5], v[8]);
  const float2 s6 = padd(v[6], v[7]);
  const float2 d6 = psub(v[6], v[7]);
  v[0] = make_float2(x0.x + (s1.x + s2.x + s3.x + s4.x + s5.x + s6.x), x0.y + (s1.y + s2.y + s3.y + s4.y + s5.y + s6.y));
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.8854560256004333f, ar); ai = fmaf(s1.y, 0.8854560256004333f, ai); br = fmaf(d1.x, 0.4647231698036194f, br); bi = fmaf(d1.y, 0.4647231698036194f, bi);
    ar = fmaf(s2.x, 0.5680647492408752f, ar); ai = fmaf(s2.y, 0.5680647492408752f, ai); br = fmaf(d2.x, 0.8229838609695435f, br); bi = fmaf(d2.y, 0.8229838609695435f, bi);
    ar = fmaf(s3.x, 0.1205366775393486f, ar); ai = fmaf(s3.y, 0.1205366775393486f, ai); br = fmaf(d3.x, 0.9927088618278503f, br); bi = fmaf(d3.y, 0.9927088618278503f, bi);
    ar = fmaf(s4.x, -0.35460489988327026f, ar); ai = fmaf(s4.y, -0.35460489988327026f, ai); br = fmaf(d4.x, 0.9350162148475647f, br); bi = fmaf(d4.y, 0.9350162148475647f, bi);
    ar = fmaf(s5.x, -0.7485107779502869f, ar); ai = fmaf(s5.y, -0.7485107779502869f, ai); br = fmaf(d5.x, 0.6631226539611816f, br); bi = fmaf(d5.y, 0.6631226539611816f, bi);
    ar = fmaf(s6.x, -0.9709418416023254f, ar); ai = fmaf(s6.y, -0.9709418416023254f, ai); br = fmaf(d6.x, 0.23931565880775452f, br); bi = fmaf(d6.y, 0.23931565880775452f, bi);
    if (!INV) {
      v[1] = make_float2(ar + bi, ai - br); v[12] = make_float2(ar - bi, ai + br);
    } else {
      v[1] = make_float2(ar - bi, ai + br); v[12] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.5680647492408752f, ar); ai = fmaf(s1.y, 0.5680647492408752f, ai); br = fmaf(d1.x, 0.8229838609695435f, br); bi = fmaf(d1.y, 0.8229838609695435f, bi);
    ar = fmaf(s2.x, -0.35460489988327026f, ar); ai = fmaf(s2.y, -0.35460489988327026f, ai); br = fmaf(d2.x, 0.9350162148475647f, br); bi = fmaf(d2.y, 0.9350162148475647f, bi);
    ar = fmaf(s3.x, -0.9709418416023254f, ar); ai = fmaf(s3.y, -0.9709418416023254f, ai); br = fmaf(d3.x, 0.23931565880775452f, br); bi = fmaf(d3.y, 0.23931565880775452f, bi);
    ar = fmaf(s4.x, -0.7485107779502869f, ar); ai = fmaf(s4.y, -0.7485107779502869f, ai); br = fmaf(d4.x, -0.6631226539611816f, br); bi = fmaf(d4.y, -0.6631226539611816f, bi);
    ar = fmaf(s5.x, 0.1205366775393486f, ar); ai = fmaf(s5.y, 0.1205366775393486f, ai); br = fmaf(d5.x, -0.9927088618278503f, br); bi = fmaf(d5.y, -0.9927088618278503f, bi);
    ar = fmaf(s6.x, 0.8854560256004333f, ar); ai = fmaf(s6.y, 0.8854560256004333f, ai); br = fmaf(d6.x, -0.4647231698036194f, br); bi = fmaf(d6.y, -0.4647231698036194f, bi);
    if (!INV) {
      v[2] = make_float2(ar + bi, ai - br); v[11] = make_float2(ar - bi, ai + br);
    } else {
      v[2] = make_float2(ar - bi, ai + br); v[11] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.1205366775393486f, ar); ai = fmaf(s1.y, 0.1205366775393486f, ai); br = fmaf(d1.x, 0.9927088618278503f, br); bi = fmaf(d1.y, 0.9927088618278503f, bi);
    ar = fmaf(s2.x, -0.9709418416023254f, ar); ai = fmaf(s2.y, -0.9709418416023254f, ai); br = fmaf(d2.x, 0.23931565880775452f, br); bi = fmaf(d2.y, 0.23931565880775452f, bi);
    ar = fmaf(s3.x, -0.35460489988327026f, ar); ai = fmaf(s3.y, -0.35460489988327026f, ai); br = fmaf(d3.x, -0.9350162148475647f, br); bi = fmaf(d3.y, -0.9350162148475647f, bi);
    ar = fmaf(s4.x, 0.8854560256004333f, ar); ai = fmaf(s4.y, 0.8854560256004333f, ai); br = fmaf(d4.x, -0.4647231698036194f, br); bi = fmaf(d4.y, -0.4647231698036194f, bi);
    ar = fmaf(s5.x, 0.5680647492408752f, ar); ai = fmaf(s5.y, 0.5680647492408752f, ai); br = fmaf(d5.x, 0.8229838609695435f, br); bi = fmaf(d5.y, 0.8229838609695435f, bi);
    ar = fmaf(s6.x, -0.7485107779502869f, ar); ai = fmaf(s6.y, -0.7485107779502869f, ai); br = fmaf(d6.x, 0.6631226539611816f, br); bi = fmaf(d6.y, 0.6631226539611816f, bi);
    if (!INV) {
      v[3] = make_float2(ar + bi, ai - br); v[10] = make_float2(ar - bi, ai + br);
    } else {
      v[3] = make_float2(ar - bi, ai + br); v[10] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.35460489988327026f, ar); ai = fmaf(s1.y, -0.35460489988327026f, ai); br = fmaf(d1.x, 0.9350162148475647f, br); bi = fmaf(d1.y, 0.9350162148475647f, bi);
    ar = fmaf(s2.x, -0.7485107779502869f, ar); ai = fmaf(s2.y, -0.7485107779502869f, ai); br = fmaf(d2.x, -0.6631226539611816f, br); bi = fmaf(d2.y, -0.6631226539611816f, bi);
    ar = fmaf(s3.x, 0.8854560256004333f, ar); ai = fmaf(s3.y, 0.8854560256004333f, ai); br = fmaf(d3.x, -0.4647231698036194f, br); bi = fmaf(d3.y, -0.4647231698036194f, bi);
    ar = fmaf(s4.x, 0.1205366775393486f, ar); ai = fmaf(s4.y, 0.1205366775393486f, ai); br = fmaf(d4.x, 0.9927088618278503f, br); bi = fmaf(d4.y, 0.9927088618278503f, bi);
    ar = fmaf(s5.x, -0.9709418416023254f, ar); ai = fmaf(s5.y, -0.9709418416023254f, ai); br = fmaf(d5.x, -0.23931565880775452f, br); bi = fmaf(d5.y, -0.23931565880775452f, bi);
    ar = fmaf(s6.x, 0.5680647492408752f, ar); ai = fmaf(s6.y, 0.5680647492408752f, ai); br = fmaf(d6.x, -0.8229838609695435f, br); bi = fmaf(d6.y, -0.8229838609695435f, bi);
    if (!INV) {
      v[4] = make_float2(ar + bi, ai - br); v[9] = make_float2(ar - bi, ai + br);
    } else {
      v[4] = make_float2(ar - bi, ai + br); v[9] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.7485107779502869f, ar); ai = fmaf(s1.y, -0.7485107779502869f, ai); br = fmaf(d1.x, 0.6631226539611816f, br); bi = fmaf(d1.y, 0.6631226539611816f, bi);
    ar = fmaf(s2.x, 0.1205366775393486f, ar); ai = fmaf(s2.y, 0.1205366775393486f, ai); br = fmaf(d2.x, -0.9927088618278503f, br); bi = fmaf(d2.y, -0.9927088618278503f, bi);
    ar = fmaf(s3.x, 0.5680647492408752f, ar); ai = fmaf(s3.y, 0.5680647492408752f, ai); br = fmaf(d3.x, 0.8229838609695435f, br); bi = fmaf(d3.y, 0.8229838609695435f, bi);
    ar = fmaf(s4.x, -0.9709418416023254f, ar); ai = fmaf(s4.y, -0.9709418416023254f, ai); br = fmaf(d4.x, -0.23931565880775452f, br); bi = fmaf(d4.y, -0.23931565880775452f, bi);
    ar = fmaf(s5.x, 0.8854560256004333f, ar); ai = fmaf(s5.y, 0.8854560256004333f, ai); br = fmaf(d5.x, -0.4647231698036194f, br); bi = fmaf(d5.y, -0.4647231698036194f, bi);
    ar = fmaf(s6.x, -0.35460489988327026f, ar); ai = fmaf(s6.y, -0.35460489988327026f, ai); br = fmaf(d6.x, 0.9350162148475647f, br); bi = fmaf(d6.y, 0.9350162148475647f, bi);
    if (!INV) {
      v[5] = make_float2(ar + bi, ai - br); v[8] = make_float2(ar - bi, ai + br);
    } else {
      v[5] = make_float2(ar - bi, ai + br); v[8] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.9709418416023254f, ar); ai = fmaf(s1.y, -0.9709418416023254f, ai); br = fmaf(d1.x, 0.23931565880775452f, br); bi = fmaf(d1.y, 0.23931565880775452f, bi);
    ar = fmaf(s2.x, 0.8854560256004333f, ar); ai = fmaf(s2.y, 0.8854560256004333f, ai); br = fmaf(d2.x, -0.4647231698036194f, br); bi = fmaf(d2.y, -0.4647231698036194f, bi);
    ar = fmaf(s3.x, -0.7485107779502869f, ar); ai = fmaf(s3.y, -0.7485107779502869f, ai); br = fmaf(d3.x, 0.6631226539611816f, br); bi = fmaf(d3.y, 0.6631226539611816f, bi);
    ar = fmaf(s4.x, 0.5680647492408752f, ar); ai = fmaf(s4.y, 0.5680647492408752f, ai); br = fmaf(d4.x, -0.8229838609695435f, br); bi = fmaf(d4.y, -0.8229838609695435f, bi);
    ar = fmaf(s5.x, -0.35460489988327026f, ar); ai = fmaf(s5.y, -0.35460489988327026f, ai); br = fmaf(d5.x, 0.9350162148475647f, br); bi = fmaf(d5.y, 0.9350162148475647f, bi);
    ar = fmaf(s6.x, 0.1205366775393486f, ar); ai = fmaf(s6.y, 0.1205366775393486f, ai); br = fmaf(d6.x, -0.9927088618278503f, br); bi = fmaf(d6.y, -0.9927088618278503f, bi);
    if (!INV) {
      v[6] = make_float2(ar + bi, ai - br); v[7] = make_float2(ar - bi, ai + br);
    } else {
      v[6] = make_float2(ar - bi, ai + br); v[7] = make_float2(ar + bi, ai - br);
    }
  }
#endif
}
template <bool INV> __device__ __forceinline__ void dft_r53(float2* v) {
  const float2 x0 = v[0];
  const float2 s1 = padd(v[1], v[52]);
  const float2 d1 = psub(v[1], v[52]);
  const float2 s2 = padd(v[2], v[51]);
  const float2 d2 = psub(v[2], v[51]);
  const float2 s3 = padd(v[3], v[50]);
  const float2 d3 = psub(v[3], v[50]);
  const float2 s4 = padd(v[4], v[49]);
  const float2 d4 = psub(v[4], v[49]);
  const float2 s5 = padd(v[5], v[48]);
  const float2 d5 = psub(v[5], v[48]);
  const float2 s6 = padd(v[6], v[47]);
  const float2 d6 = psub(v[6], v[47]);
  const float2 s7 = padd(v[7], v[46]);
  const float2 d7 = psub(v[7], v[46]);
  const float2 s8 = padd(v[8], v[45]);
  const float2 d8 = psub(v[8], v[45]);
  const float2 s9 = padd(v[9], v[44]);
  const float2 d9 = psub(v[9], v[44]);
  const float2 s10 = padd(v[10], v[43]);
  const float2 d10 = psub(v[10], v[43]);
  const float2 s11 = padd(v[11], v[42]);
  const float2 d11 = psub(v[11], v[42]);
  const float2 s12 = padd(v[12], v[41]);
  const float2 d12 = psub(v[12], v[41]);
  const float2 s13 = padd(v[13], v[40]);
  const float2 d13 = psub(v[13], v[40]);
  const float2 s14 = padd(v[14], v[39]);
  const float2 d14 = psub(v[14], v[39]);
  const float2 s15 = padd(v[15], v[38]);
  const float2 d15 = psub(v[15], v[38]);
  const float2 s16 = padd(v[16], v[37]);
  const float2 d16 = psub(v[16], v[37]);
  const float2 s17 = padd(v[17], v[36]);
  const float2 d17 = psub(v[17], v[36]);
  const float2 s18 = padd(v[18], v[35]);
  const float2 d18 = psub(v[18], v[35]);
  const float2 s19 = padd(v[19], v[34]);
  const float2 d19 = psub(v[19], v[34]);
  const float2 s20 = padd(v[20], v[33]);
  const float2 d20 = psub(v[20], v[33]);
  const float2 s21 = padd(v[21], v[32]);
  const float2 d21 = psub(v[21], v[32]);
  const float2 s22 = padd(v[22], v[31]);
  const float2 d22 = psub(v[22], v[31]);
  const float2 s23 = padd(v[23], v[30]);
  const float2 d23 = psub(v[23], v[30]);
  const float2 s24 = padd(v[24], v[29]);
  const float2 d24 = psub(v[24], v[29]);
  const float2 s25 = padd(v[25], v[28]);
  const float2 d25 = psub(v[25], v[28]);
  const float2 s26 = padd(v[26], v[27]);
  const float2 d26 = psub(v[26], v[27]);
  v[0] = make_float2(x0.x + (s1.x + s2.x + s3.x + s4.x + s5.x + s6.x + s7.x + s8.x + s9.x + s10.x + s11.x + s12.x + s13.x + s14.x + s15.x + s16.x + s17.x + s18.x + s19.x + s20.x + s21.x + s22.x + s23.x + s24.x + s25.x + s26.x), x0.y + (s1.y + s2.y + s3.y + s4.y + s5.y + s6.y + s7.y + s8.y + s9.y + s10.y + s11.y + s12.y + s13.y + s14.y + s15.y + s16.y + s17.y + s18.y + s19.y + s20.y + s21.y + s22.y + s23.y + s24.y + s25.y + s26.y));
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.9929810762405396f, ar); ai = fmaf(s1.y, 0.9929810762405396f, ai); br = fmaf(d1.x, 0.11827316880226135f, br); bi = fmaf(d1.y, 0.11827316880226135f, bi);
    ar = fmaf(s2.x, 0.9720228910446167f, ar); ai = fmaf(s2.y, 0.9720228910446167f, ai); br = fmaf(d2.x, 0.2348860502243042f, br); bi = fmaf(d2.y, 0.2348860502243042f, bi);
    ar = fmaf(s3.x, 0.9374196529388428f, ar); ai = fmaf(s3.y, 0.9374196529388428f, ai); br = fmaf(d3.x, 0.3482016324996948f, br); bi = fmaf(d3.y, 0.3482016324996948f, bi);
    ar = fmaf(s4.x, 0.8896570801734924f, ar); ai = fmaf(s4.y, 0.8896570801734924f, ai); br = fmaf(d4.x, 0.4566292464733124f, br); bi = fmaf(d4.y, 0.4566292464733124f, bi);
    ar = fmaf(s5.x, 0.829405665397644f, ar); ai = fmaf(s5.y, 0.829405665397644f, ai); br = fmaf(d5.x, 0.5586467385292053f, br); bi = fmaf(d5.y, 0.5586467385292053f, bi);
    ar = fmaf(s6.x, 0.7575112581253052f, ar); ai = fmaf(s6.y, 0.7575112581253052f, ai); br = fmaf(d6.x, 0.6528221368789673f, br); bi = fmaf(d6.y, 0.6528221368789673f, bi);
    ar = fmaf(s7.x, 0.674983024597168f, ar); ai = fmaf(s7.y, 0.674983024597168f, ai); br = fmaf(d7.x, 0.7378332614898682f, br); bi = fmaf(d7.y, 0.7378332614898682f, bi);
    ar = fmaf(s8.x, 0.5829795002937317f, ar); ai = fmaf(s8.y, 0.5829795002937317f, ai); br = fmaf(d8.x, 0.8124868869781494f, br); bi = fmaf(d8.y, 0.8124868869781494f, bi);
    ar = fmaf(s9.x, 0.4827921986579895f, ar); ai = fmaf(s9.y, 0.4827921986579895f, ai); br = fmaf(d9.x, 0.8757349252700806f, br); bi = fmaf(d9.y, 0.8757349252700806f, bi);
    ar = fmaf(s10.x, 0.3758275806903839f, ar); ai = fmaf(s10.y, 0.3758275806903839f, ai); br = fmaf(d10.x, 0.926689624786377f, br); bi = fmaf(d10.y, 0.926689624786377f, bi);
    ar = fmaf(s11.x, 0.26358717679977417f, ar); ai = fmaf(s11.y, 0.26358717679977417f, ai); br = fmaf(d11.x, 0.9646356105804443f, br); bi = fmaf(d11.y, 0.9646356105804443f, bi);
    ar = fmaf(s12.x, 0.14764656126499176f, ar); ai = fmaf(s12.y, 0.14764656126499176f, ai); br = fmaf(d12.x, 0.989040195941925f, br); bi = fmaf(d12.y, 0.989040195941925f, bi);
    ar = fmaf(s13.x, 0.029633328318595886f, ar); ai = fmaf(s13.y, 0.029633328318595886f, ai); br = fmaf(d13.x, 0.9995608329772949f, br); bi = fmaf(d13.y, 0.9995608329772949f, bi);
    ar = fmaf(s14.x, -0.08879589289426804f, ar); ai = fmaf(s14.y, -0.08879589289426804f, ai); br = fmaf(d14.x, 0.9960498213768005f, br); bi = fmaf(d14.y, 0.9960498213768005f, bi);
    ar = fmaf(s15.x, -0.2059786170721054f, ar); ai = fmaf(s15.y, -0.2059786170721054f, ai); br = fmaf(d15.x, 0.9785565137863159f, br); bi = fmaf(d15.y, 0.9785565137863159f, bi);
    ar = fmaf(s16.x, -0.3202698528766632f, ar); ai = fmaf(s16.y, -0.3202698528766632f, ai); br = fmaf(d16.x, 0.9473263621330261f, br); bi = fmaf(d16.y, 0.9473263621330261f, bi);
    ar = fmaf(s17.x, -0.43006521463394165f, ar); ai = fmaf(s17.y, -0.43006521463394165f, ai); br = fmaf(d17.x, 0.9027978181838989f, br); bi = fmaf(d17.y, 0.9027978181838989f, bi);
    ar = fmaf(s18.x, -0.5338233709335327f, ar); ai = fmaf(s18.y, -0.5338233709335327f, ai); br = fmaf(d18.x, 0.8455960154533386f, br); bi = fmaf(d18.y, 0.8455960154533386f, bi);
    ar = fmaf(s19.x, -0.6300878524780273f, ar); ai = fmaf(s19.y, -0.6300878524780273f, ai); br = fmaf(d19.x, 0.7765238881111145f, br); bi = fmaf(d19.y, 0.7765238881111145f, bi);
    ar = fmaf(s20.x, -0.7175072431564331f, ar); ai = fmaf(s20.y, -0.7175072431564331f, ai); br = fmaf(d20.x, 0.6965510249137878f, br); bi = fmaf(d20.y, 0.6965510249137878f, bi);
    ar = fmaf(s21.x, -0.794854462146759f, ar); ai = fmaf(s21.y, -0.794854462146759f, ai); br = fmaf(d21.x, 0.6068001389503479f, br); bi = fmaf(d21.y, 0.6068001389503479f, bi);
    ar = fmaf(s22.x, -0.8610436320304871f, ar); ai = fmaf(s22.y, -0.8610436320304871f, ai); br = fmaf(d22.x, 0.5085310935974121f, br); bi = fmaf(d22.y, 0.5085310935974121f, bi);
    ar = fmaf(s23.x, -0.9151456356048584f, ar); ai = fmaf(s23.y, -0.9151456356048584f, ai); br = fmaf(d23.x, 0.4031234383583069f, br); bi = fmaf(d23.y, 0.4031234383583069f, bi);
    ar = fmaf(s24.x, -0.956400990486145f, ar); ai = fmaf(s24.y, -0.956400990486145f, ai); br = fmaf(d24.x, 0.29205676913261414f, br); bi = fmaf(d24.y, 0.29205676913261414f, bi);
    ar = fmaf(s25.x, -0.9842305779457092f, ar); ai = fmaf(s25.y, -0.9842305779457092f, ai); br = fmaf(d25.x, 0.1768902689218521f, br); bi = fmaf(d25.y, 0.1768902689218521f, bi);
    ar = fmaf(s26.x, -0.9982437491416931f, ar); ai = fmaf(s26.y, -0.9982437491416931f, ai); br = fmaf(d26.x, 0.05924062803387642f, br); bi = fmaf(d26.y, 0.05924062803387642f, bi);
    if (!INV) {
      v[1] = make_float2(ar + bi, ai - br); v[52] = make_float2(ar - bi, ai + br);
    } else {
      v[1] = make_float2(ar - bi, ai + br); v[52] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.9720228910446167f, ar); ai = fmaf(s1.y, 0.9720228910446167f, ai); br = fmaf(d1.x, 0.2348860502243042f, br); bi = fmaf(d1.y, 0.2348860502243042f, bi);
    ar = fmaf(s2.x, 0.8896570801734924f, ar); ai = fmaf(s2.y, 0.8896570801734924f, ai); br = fmaf(d2.x, 0.4566292464733124f, br); bi = fmaf(d2.y, 0.4566292464733124f, bi);
    ar = fmaf(s3.x, 0.7575112581253052f, ar); ai = fmaf(s3.y, 0.7575112581253052f, ai); br = fmaf(d3.x, 0.6528221368789673f, br); bi = fmaf(d3.y, 0.6528221368789673f, bi);
    ar = fmaf(s4.x, 0.5829795002937317f, ar); ai = fmaf(s4.y, 0.5829795002937317f, ai); br = fmaf(d4.x, 0.8124868869781494f, br); bi = fmaf(d4.y, 0.8124868869781494f, bi);
    ar = fmaf(s5.x, 0.3758275806903839f, ar); ai = fmaf(s5.y, 0.3758275806903839f, ai); br = fmaf(d5.x, 0.926689624786377f, br); bi = fmaf(d5.y, 0.926689624786377f, bi);
    ar = fmaf(s6.x, 0.14764656126499176f, ar); ai = fmaf(s6.y, 0.14764656126499176f, ai); br = fmaf(d6.x, 0.989040195941925f, br); bi = fmaf(d6.y, 0.989040195941925f, bi);
    ar = fmaf(s7.x, -0.08879589289426804f, ar); ai = fmaf(s7.y, -0.08879589289426804f, ai); br = fmaf(d7.x, 0.9960498213768005f, br); bi = fmaf(d7.y, 0.9960498213768005f, bi);
    ar = fmaf(s8.x, -0.3202698528766632f, ar); ai = fmaf(s8.y, -0.3202698528766632f, ai); br = fmaf(d8.x, 0.9473263621330261f, br); bi = fmaf(d8.y, 0.9473263621330261f, bi);
    ar = fmaf(s9.x, -0.5338233709335327f, ar); ai = fmaf(s9.y, -0.5338233709335327f, ai); br = fmaf(d9.x, 0.8455960154533386f, br); bi = fmaf(d9.y, 0.8455960154533386f, bi);
    ar = fmaf(s10.x, -0.7175072431564331f, ar); ai = fmaf(s10.y, -0.7175072431564331f, ai); br = fmaf(d10.x, 0.6965510249137878f, br); bi = fmaf(d10.y, 0.6965510249137878f, bi);
    ar = fmaf(s11.x, -0.8610436320304871f, ar); ai = fmaf(s11.y, -0.8610436320304871f, ai); br = fmaf(d11.x, 0.5085310935974121f, br); bi = fmaf(d11.y, 0.5085310935974121f, bi);
    ar = fmaf(s12.x, -0.956400990486145f, ar); ai = fmaf(s12.y, -0.956400990486145f, ai); br = fmaf(d12.x, 0.29205676913261414f, br); bi = fmaf(d12.y, 0.29205676913261414f, bi);
    ar = fmaf(s13.x, -0.9982437491416931f, ar); ai = fmaf(s13.y, -0.9982437491416931f, ai); br = fmaf(d13.x, 0.05924062803387642f, br); bi = fmaf(d13.y, 0.05924062803387642f, bi);
    ar = fmaf(s14.x, -0.9842305779457092f, ar); ai = fmaf(s14.y, -0.9842305779457092f, ai); br = fmaf(d14.x, -0.1768902689218521f, br); bi = fmaf(d14.y, -0.1768902689218521f, bi);
    ar = fmaf(s15.x, -0.9151456356048584f, ar); ai = fmaf(s15.y, -0.9151456356048584f, ai); br = fmaf(d15.x, -0.4031234383583069f, br); bi = fmaf(d15.y, -0.4031234383583069f, bi);
    ar = fmaf(s16.x, -0.794854462146759f, ar); ai = fmaf(s16.y, -0.794854462146759f, ai); br = fmaf(d16.x, -0.6068001389503479f, br); bi = fmaf(d16.y, -0.6068001389503479f, bi);
    ar = fmaf(s17.x, -0.6300878524780273f, ar); ai = fmaf(s17.y, -0.6300878524780273f, ai); br = fmaf(d17.x, -0.7765238881111145f, br); bi = fmaf(d17.y, -0.7765238881111145f, bi);
    ar = fmaf(s18.x, -0.43006521463394165f, ar); ai = fmaf(s18.y, -0.43006521463394165f, ai); br = fmaf(d18.x, -0.9027978181838989f, br); bi = fmaf(d18.y, -0.9027978181838989f, bi);
    ar = fmaf(s19.x, -0.2059786170721054f, ar); ai = fmaf(s19.y, -0.2059786170721054f, ai); br = fmaf(d19.x, -0.9785565137863159f, br); bi = fmaf(d19.y, -0.9785565137863159f, bi);
    ar = fmaf(s20.x, 0.029633328318595886f, ar); ai = fmaf(s20.y, 0.029633328318595886f, ai); br = fmaf(d20.x, -0.9995608329772949f, br); bi = fmaf(d20.y, -0.9995608329772949f, bi);
    ar = fmaf(s21.x, 0.26358717679977417f, ar); ai = fmaf(s21.y, 0.26358717679977417f, ai); br = fmaf(d21.x, -0.9646356105804443f, br); bi = fmaf(d21.y, -0.9646356105804443f, bi);
    ar = fmaf(s22.x, 0.4827921986579895f, ar); ai = fmaf(s22.y, 0.4827921986579895f, ai); br = fmaf(d22.x, -0.8757349252700806f, br); bi = fmaf(d22.y, -0.8757349252700806f, bi);
    ar = fmaf(s23.x, 0.674983024597168f, ar); ai = fmaf(s23.y, 0.674983024597168f, ai); br = fmaf(d23.x, -0.7378332614898682f, br); bi = fmaf(d23.y, -0.7378332614898682f, bi);
    ar = fmaf(s24.x, 0.829405665397644f, ar); ai = fmaf(s24.y, 0.829405665397644f, ai); br = fmaf(d24.x, -0.5586467385292053f, br); bi = fmaf(d24.y, -0.5586467385292053f, bi);
    ar = fmaf(s25.x, 0.9374196529388428f, ar); ai = fmaf(s25.y, 0.9374196529388428f, ai); br = fmaf(d25.x, -0.3482016324996948f, br); bi = fmaf(d25.y, -0.3482016324996948f, bi);
    ar = fmaf(s26.x, 0.9929810762405396f, ar); ai = fmaf(s26.y, 0.9929810762405396f, ai); br = fmaf(d26.x, -0.11827316880226135f, br); bi = fmaf(d26.y, -0.11827316880226135f, bi);
    if (!INV) {
      v[2] = make_float2(ar + bi, ai - br); v[51] = make_float2(ar - bi, ai + br);
    } else {
      v[2] = make_float2(ar - bi, ai + br); v[51] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.9374196529388428f, ar); ai = fmaf(s1.y, 0.9374196529388428f, ai); br = fmaf(d1.x, 0.3482016324996948f, br); bi = fmaf(d1.y, 0.3482016324996948f, bi);
    ar = fmaf(s2.x, 0.7575112581253052f, ar); ai = fmaf(s2.y, 0.7575112581253052f, ai); br = fmaf(d2.x, 0.6528221368789673f, br); bi = fmaf(d2.y, 0.6528221368789673f, bi);
    ar = fmaf(s3.x, 0.4827921986579895f, ar); ai = fmaf(s3.y, 0.4827921986579895f, ai); br = fmaf(d3.x, 0.8757349252700806f, br); bi = fmaf(d3.y, 0.8757349252700806f, bi);
    ar = fmaf(s4.x, 0.14764656126499176f, ar); ai = fmaf(s4.y, 0.14764656126499176f, ai); br = fmaf(d4.x, 0.989040195941925f, br); bi = fmaf(d4.y, 0.989040195941925f, bi);
    ar = fmaf(s5.x, -0.2059786170721054f, ar); ai = fmaf(s5.y, -0.2059786170721054f, ai); br = fmaf(d5.x, 0.9785565137863159f, br); bi = fmaf(d5.y, 0.9785565137863159f, bi);
    ar = fmaf(s6.x, -0.5338233709335327f, ar); ai = fmaf(s6.y, -0.5338233709335327f, ai); br = fmaf(d6.x, 0.8455960154533386f, br); bi = fmaf(d6.y, 0.8455960154533386f, bi);
    ar = fmaf(s7.x, -0.794854462146759f, ar); ai = fmaf(s7.y, -0.794854462146759f, ai); br = fmaf(d7.x, 0.6068001389503479f, br); bi = fmaf(d7.y, 0.6068001389503479f, bi);
    ar = fmaf(s8.x, -0.956400990486145f, ar); ai = fmaf(s8.y, -0.956400990486145f, ai); br = fmaf(d8.x, 0.29205676913261414f, br); bi = fmaf(d8.y, 0.29205676913261414f, bi);
    ar = fmaf(s9.x, -0.9982437491416931f, ar); ai = fmaf(s9.y, -0.9982437491416931f, ai); br = fmaf(d9.x, -0.05924062803387642f, br); bi = fmaf(d9.y, -0.05924062803387642f, bi);
    ar = fmaf(s10.x, -0.9151456356048584f, ar); ai = fmaf(s10.y, -0.9151456356048584f, ai); br = fmaf(d10.x, -0.4031234383583069f, br); bi = fmaf(d10.y, -0.4031234383583069f, bi);
    ar = fmaf(s11.x, -0.7175072431564331f, ar); ai = fmaf(s11.y, -0.7175072431564331f, ai); br = fmaf(d11.x, -0.6965510249137878f, br); bi = fmaf(d11.y, -0.6965510249137878f, bi);
    ar = fmaf(s12.x, -0.43006521463394165f, ar); ai = fmaf(s12.y, -0.43006521463394165f, ai); br = fmaf(d12.x, -0.9027978181838989f, br); bi = fmaf(d12.y, -0.9027978181838989f, bi);
    ar = fmaf(s13.x, -0.08879589289426804f, ar); ai = fmaf(s13.y, -0.08879589289426804f, ai); br = fmaf(d13.x, -0.9960498213768005f, br); bi = fmaf(d13.y, -0.9960498213768005f, bi);
    ar = fmaf(s14.x, 0.26358717679977417f, ar); ai = fmaf(s14.y, 0.26358717679977417f, ai); br = fmaf(d14.x, -0.9646356105804443f, br); bi = fmaf(d14.y, -0.9646356105804443f, bi);
    ar = fmaf(s15.x, 0.5829795002937317f, ar); ai = fmaf(s15.y, 0.5829795002937317f, ai); br = fmaf(d15.x, -0.8124868869781494f, br); bi = fmaf(d15.y, -0.8124868869781494f, bi);
    ar = fmaf(s16.x, 0.829405665397644f, ar); ai = fmaf(s16.y, 0.829405665397644f, ai); br = fmaf(d16.x, -0.5586467385292053f, br); bi = fmaf(d16.y, -0.5586467385292053f, bi);
    ar = fmaf(s17.x, 0.9720228910446167f, ar); ai = fmaf(s17.y, 0.9720228910446167f, ai); br = fmaf(d17.x, -0.2348860502243042f, br); bi = fmaf(d17.y, -0.2348860502243042f, bi);
    ar = fmaf(s18.x, 0.9929810762405396f, ar); ai = fmaf(s18.y, 0.9929810762405396f, ai); br = fmaf(d18.x, 0.11827316880226135f, br); bi = fmaf(d18.y, 0.11827316880226135f, bi);
    ar = fmaf(s19.x, 0.8896570801734924f, ar); ai = fmaf(s19.y, 0.8896570801734924f, ai); br = fmaf(d19.x, 0.4566292464733124f, br); bi = fmaf(d19.y, 0.4566292464733124f, bi);
    ar = fmaf(s20.x, 0.674983024597168f, ar); ai = fmaf(s20.y, 0.674983024597168f, ai); br = fmaf(d20.x, 0.7378332614898682f, br); bi = fmaf(d20.y, 0.7378332614898682f, bi);
    ar = fmaf(s21.x, 0.3758275806903839f, ar); ai = fmaf(s21.y, 0.3758275806903839f, ai); br = fmaf(d21.x, 0.926689624786377f, br); bi = fmaf(d21.y, 0.926689624786377f, bi);
    ar = fmaf(s22.x, 0.029633328318595886f, ar); ai = fmaf(s22.y, 0.029633328318595886f, ai); br = fmaf(d22.x, 0.9995608329772949f, br); bi = fmaf(d22.y, 0.9995608329772949f, bi);
    ar = fmaf(s23.x, -0.3202698528766632f, ar); ai = fmaf(s23.y, -0.3202698528766632f, ai); br = fmaf(d23.x, 0.9473263621330261f, br); bi = fmaf(d23.y, 0.9473263621330261f, bi);
    ar = fmaf(s24.x, -0.6300878524780273f, ar); ai = fmaf(s24.y, -0.6300878524780273f, ai); br = fmaf(d24.x, 0.7765238881111145f, br); bi = fmaf(d24.y, 0.7765238881111145f, bi);
    ar = fmaf(s25.x, -0.8610436320304871f, ar); ai = fmaf(s25.y, -0.8610436320304871f, ai); br = fmaf(d25.x, 0.5085310935974121f, br); bi = fmaf(d25.y, 0.5085310935974121f, bi);
    ar = fmaf(s26.x, -0.9842305779457092f, ar); ai = fmaf(s26.y, -0.9842305779457092f, ai); br = fmaf(d26.x, 0.1768902689218521f, br); bi = fmaf(d26.y, 0.1768902689218521f, bi);
    if (!INV) {
      v[3] = make_float2(ar + bi, ai - br); v[50] = make_float2(ar - bi, ai + br);
    } else {
      v[3] = make_float2(ar - bi, ai + br); v[50] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.8896570801734924f, ar); ai = fmaf(s1.y, 0.8896570801734924f, ai); br = fmaf(d1.x, 0.4566292464733124f, br); bi = fmaf(d1.y, 0.4566292464733124f, bi);
    ar = fmaf(s2.x, 0.5829795002937317f, ar); ai = fmaf(s2.y, 0.5829795002937317f, ai); br = fmaf(d2.x, 0.8124868869781494f, br); bi = fmaf(d2.y, 0.8124868869781494f, bi);
    ar = fmaf(s3.x, 0.14764656126499176f, ar); ai = fmaf(s3.y, 0.14764656126499176f, ai); br = fmaf(d3.x, 0.989040195941925f, br); bi = fmaf(d3.y, 0.989040195941925f, bi);
    ar = fmaf(s4.x, -0.3202698528766632f, ar); ai = fmaf(s4.y, -0.3202698528766632f, ai); br = fmaf(d4.x, 0.9473263621330261f, br); bi = fmaf(d4.y, 0.9473263621330261f, bi);
    ar = fmaf(s5.x, -0.7175072431564331f, ar); ai = fmaf(s5.y, -0.7175072431564331f, ai); br = fmaf(d5.x, 0.6965510249137878f, br); bi = fmaf(d5.y, 0.6965510249137878f, bi);
    ar = fmaf(s6.x, -0.956400990486145f, ar); ai = fmaf(s6.y, -0.956400990486145f, ai); br = fmaf(d6.x, 0.29205676913261414f, br); bi = fmaf(d6.y, 0.29205676913261414f, bi);
    ar = fmaf(s7.x, -0.9842305779457092f, ar); ai = fmaf(s7.y, -0.9842305779457092f, ai); br = fmaf(d7.x, -0.1768902689218521f, br); bi = fmaf(d7.y, -0.1768902689218521f, bi);
    ar = fmaf(s8.x, -0.794854462146759f, ar); ai = fmaf(s8.y, -0.794854462146759f, ai); br = fmaf(d8.x, -0.6068001389503479f, br); bi = fmaf(d8.y, -0.6068001389503479f, bi);
    ar = fmaf(s9.x, -0.43006521463394165f, ar); ai = fmaf(s9.y, -0.43006521463394165f, ai); br = fmaf(d9.x, -0.9027978181838989f, br); bi = fmaf(d9.y, -0.9027978181838989f, bi);
    ar = fmaf(s10.x, 0.029633328318595886f, ar); ai = fmaf(s10.y, 0.029633328318595886f, ai); br = fmaf(d10.x, -0.9995608329772949f, br); bi = fmaf(d10.y, -0.9995608329772949f, bi);
    ar = fmaf(s11.x, 0.4827921986579895f, ar); ai = fmaf(s11.y, 0.4827921986579895f, ai); br = fmaf(d11.x, -0.8757349252700806f, br); bi = fmaf(d11.y, -0.8757349252700806f, bi);
    ar = fmaf(s12.x, 0.829405665397644f, ar); ai = fmaf(s12.y, 0.829405665397644f, ai); br = fmaf(d12.x, -0.5586467385292053f, br); bi = fmaf(d12.y, -0.5586467385292053f, bi);
    ar = fmaf(s13.x, 0.9929810762405396f, ar); ai = fmaf(s13.y, 0.9929810762405396f, ai); br = fmaf(d13.x, -0.11827316880226135f, br); bi = fmaf(d13.y, -0.11827316880226135f, bi);
    ar = fmaf(s14.x, 0.9374196529388428f, ar); ai = fmaf(s14.y, 0.9374196529388428f, ai); br = fmaf(d14.x, 0.3482016324996948f, br); bi = fmaf(d14.y, 0.3482016324996948f, bi);
    ar = fmaf(s15.x, 0.674983024597168f, ar); ai = fmaf(s15.y, 0.674983024597168f, ai); br = fmaf(d15.x, 0.7378332614898682f, br); bi = fmaf(d15.y, 0.7378332614898682f, bi);
    ar = fmaf(s16.x, 0.26358717679977417f, ar); ai = fmaf(s16.y, 0.26358717679977417f, ai); br = fmaf(d16.x, 0.9646356105804443f, br); bi = fmaf(d16.y, 0.9646356105804443f, bi);
    ar = fmaf(s17.x, -0.2059786170721054f, ar); ai = fmaf(s17.y, -0.2059786170721054f, ai); br = fmaf(d17.x, 0.9785565137863159f, br); bi = fmaf(d17.y, 0.9785565137863159f, bi);
    ar = fmaf(s18.x, -0.6300878524780273f, ar); ai = fmaf(s18.y, -0.6300878524780273f, ai); br = fmaf(d18.x, 0.7765238881111145f, br); bi = fmaf(d18.y, 0.7765238881111145f, bi);
    ar = fmaf(s19.x, -0.9151456356048584f, ar); ai = fmaf(s19.y, -0.9151456356048584f, ai); br = fmaf(d19.x, 0.4031234383583069f, br); bi = fmaf(d19.y, 0.4031234383583069f, bi);
    ar = fmaf(s20.x, -0.9982437491416931f, ar); ai = fmaf(s20.y, -0.9982437491416931f, ai); br = fmaf(d20.x, -0.05924062803387642f, br); bi = fmaf(d20.y, -0.05924062803387642f, bi);
    ar = fmaf(s21.x, -0.8610436320304871f, ar); ai = fmaf(s21.y, -0.8610436320304871f, ai); br = fmaf(d21.x, -0.5085310935974121f, br); bi = fmaf(d21.y, -0.5085310935974121f, bi);
    ar = fmaf(s22.x, -0.5338233709335327f, ar); ai = fmaf(s22.y, -0.5338233709335327f, ai); br = fmaf(d22.x, -0.8455960154533386f, br); bi = fmaf(d22.y, -0.8455960154533386f, bi);
    ar = fmaf(s23.x, -0.08879589289426804f, ar); ai = fmaf(s23.y, -0.08879589289426804f, ai); br = fmaf(d23.x, -0.9960498213768005f, br); bi = fmaf(d23.y, -0.9960498213768005f, bi);
    ar = fmaf(s24.x, 0.3758275806903839f, ar); ai = fmaf(s24.y, 0.3758275806903839f, ai); br = fmaf(d24.x, -0.926689624786377f, br); bi = fmaf(d24.y, -0.926689624786377f, bi);
    ar = fmaf(s25.x, 0.7575112581253052f, ar); ai = fmaf(s25.y, 0.7575112581253052f, ai); br = fmaf(d25.x, -0.6528221368789673f, br); bi = fmaf(d25.y, -0.6528221368789673f, bi);
    ar = fmaf(s26.x, 0.9720228910446167f, ar); ai = fmaf(s26.y, 0.9720228910446167f, ai); br = fmaf(d26.x, -0.2348860502243042f, br); bi = fmaf(d26.y, -0.2348860502243042f, bi);
    if (!INV) {
      v[4] = make_float2(ar + bi, ai - br); v[49] = make_float2(ar - bi, ai + br);
    } else {
      v[4] = make_float2(ar - bi, ai + br); v[49] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.829405665397644f, ar); ai = fmaf(s1.y, 0.829405665397644f, ai); br = fmaf(d1.x, 0.5586467385292053f, br); bi = fmaf(d1.y, 0.5586467385292053f, bi);
    ar = fmaf(s2.x, 0.3758275806903839f, ar); ai = fmaf(s2.y, 0.3758275806903839f, ai); br = fmaf(d2.x, 0.926689624786377f, br); bi = fmaf(d2.y, 0.926689624786377f, bi);
    ar = fmaf(s3.x, -0.2059786170721054f, ar); ai = fmaf(s3.y, -0.2059786170721054f, ai); br = fmaf(d3.x, 0.9785565137863159f, br); bi = fmaf(d3.y, 0.9785565137863159f, bi);
    ar = fmaf(s4.x, -0.7175072431564331f, ar); ai = fmaf(s4.y, -0.7175072431564331f, ai); br = fmaf(d4.x, 0.6965510249137878f, br); bi = fmaf(d4.y, 0.6965510249137878f, bi);
    ar = fmaf(s5.x, -0.9842305779457092f, ar); ai = fmaf(s5.y, -0.9842305779457092f, ai); br = fmaf(d5.x, 0.1768902689218521f, br); bi = fmaf(d5.y, 0.1768902689218521f, bi);
    ar = fmaf(s6.x, -0.9151456356048584f, ar); ai = fmaf(s6.y, -0.9151456356048584f, ai); br = fmaf(d6.x, -0.4031234383583069f, br); bi = fmaf(d6.y, -0.4031234383583069f, bi);
    ar = fmaf(s7.x, -0.5338233709335327f, ar); ai = fmaf(s7.y, -0.5338233709335327f, ai); br = fmaf(d7.x, -0.8455960154533386f, br); bi = fmaf(d7.y, -0.8455960154533386f, bi);
    ar = fmaf(s8.x, 0.029633328318595886f, ar); ai = fmaf(s8.y, 0.029633328318595886f, ai); br = fmaf(d8.x, -0.9995608329772949f, br); bi = fmaf(d8.y, -0.9995608329772949f, bi);
    ar = fmaf(s9.x, 0.5829795002937317f, ar); ai = fmaf(s9.y, 0.5829795002937317f, ai); br = fmaf(d9.x, -0.8124868869781494f, br); bi = fmaf(d9.y, -0.8124868869781494f, bi);
    ar = fmaf(s10.x, 0.9374196529388428f, ar); ai = fmaf(s10.y, 0.9374196529388428f, ai); br = fmaf(d10.x, -0.3482016324996948f, br); bi = fmaf(d10.y, -0.3482016324996948f, bi);
    ar = fmaf(s11.x, 0.9720228910446167f, ar); ai = fmaf(s11.y, 0.9720228910446167f, ai); br = fmaf(d11.x, 0.2348860502243042f, br); bi = fmaf(d11.y, 0.2348860502243042f, bi);
    ar = fmaf(s12.x, 0.674983024597168f, ar); ai = fmaf(s12.y, 0.674983024597168f, ai); br = fmaf(d12.x, 0.7378332614898682f, br); bi = fmaf(d12.y, 0.7378332614898682f, bi);
    ar = fmaf(s13.x, 0.14764656126499176f, ar); ai = fmaf(s13.y, 0.14764656126499176f, ai); br = fmaf(d13.x, 0.989040195941925f, br); bi = fmaf(d13.y, 0.989040195941925f, bi);
    ar = fmaf(s14.x, -0.43006521463394165f, ar); ai = fmaf(s14.y, -0.43006521463394165f, ai); br = fmaf(d14.x, 0.9027978181838989f, br); bi = fmaf(d14.y, 0.9027978181838989f, bi);
    ar = fmaf(s15.x, -0.8610436320304871f, ar); ai = fmaf(s15.y, -0.8610436320304871f, ai); br = fmaf(d15.x, 0.5085310935974121f, br); bi = fmaf(d15.y, 0.5085310935974121f, bi);
    ar = fmaf(s16.x, -0.9982437491416931f, ar); ai = fmaf(s16.y, -0.9982437491416931f, ai); br = fmaf(d16.x, -0.05924062803387642f, br); bi = fmaf(d16.y, -0.05924062803387642f, bi);
    ar = fmaf(s17.x, -0.794854462146759f, ar); ai = fmaf(s17.y, -0.794854462146759f, ai); br = fmaf(d17.x, -0.6068001389503479f, br); bi = fmaf(d17.y, -0.6068001389503479f, bi);
    ar = fmaf(s18.x, -0.3202698528766632f, ar); ai = fmaf(s18.y, -0.3202698528766632f, ai); br = fmaf(d18.x, -0.9473263621330261f, br); bi = fmaf(d18.y, -0.9473263621330261f, bi);
    ar = fmaf(s19.x, 0.26358717679977417f, ar); ai = fmaf(s19.y, 0.26358717679977417f, ai); br = fmaf(d19.x, -0.9646356105804443f, br); bi = fmaf(d19.y, -0.9646356105804443f, bi);
    ar = fmaf(s20.x, 0.7575112581253052f, ar); ai = fmaf(s20.y, 0.7575112581253052f, ai); br = fmaf(d20.x, -0.6528221368789673f, br); bi = fmaf(d20.y, -0.6528221368789673f, bi);
    ar = fmaf(s21.x, 0.9929810762405396f, ar); ai = fmaf(s21.y, 0.9929810762405396f, ai); br = fmaf(d21.x, -0.11827316880226135f, br); bi = fmaf(d21.y, -0.11827316880226135f, bi);
    ar = fmaf(s22.x, 0.8896570801734924f, ar); ai = fmaf(s22.y, 0.8896570801734924f, ai); br = fmaf(d22.x, 0.4566292464733124f, br); bi = fmaf(d22.y, 0.4566292464733124f, bi);
    ar = fmaf(s23.x, 0.4827921986579895f, ar); ai = fmaf(s23.y, 0.4827921986579895f, ai); br = fmaf(d23.x, 0.8757349252700806f, br); bi = fmaf(d23.y, 0.8757349252700806f, bi);
    ar = fmaf(s24.x, -0.08879589289426804f, ar); ai = fmaf(s24.y, -0.08879589289426804f, ai); br = fmaf(d24.x, 0.9960498213768005f, br); bi = fmaf(d24.y, 0.9960498213768005f, bi);
    ar = fmaf(s25.x, -0.6300878524780273f, ar); ai = fmaf(s25.y, -0.6300878524780273f, ai); br = fmaf(d25.x, 0.7765238881111145f, br); bi = fmaf(d25.y, 0.7765238881111145f, bi);
    ar = fmaf(s26.x, -0.956400990486145f, ar); ai = fmaf(s26.y, -0.956400990486145f, ai); br = fmaf(d26.x, 0.29205676913261414f, br); bi = fmaf(d26.y, 0.29205676913261414f, bi);
    if (!INV) {
      v[5] = make_float2(ar + bi, ai - br); v[48] = make_float2(ar - bi, ai + br);
    } else {
      v[5] = make_float2(ar - bi, ai + br); v[48] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.7575112581253052f, ar); ai = fmaf(s1.y, 0.7575112581253052f, ai); br = fmaf(d1.x, 0.6528221368789673f, br); bi = fmaf(d1.y, 0.6528221368789673f, bi);
    ar = fmaf(s2.x, 0.14764656126499176f, ar); ai = fmaf(s2.y, 0.14764656126499176f, ai); br = fmaf(d2.x, 0.989040195941925f, br); bi = fmaf(d2.y, 0.989040195941925f, bi);
    ar = fmaf(s3.x, -0.5338233709335327f, ar); ai = fmaf(s3.y, -0.5338233709335327f, ai); br = fmaf(d3.x, 0.8455960154533386f, br); bi = fmaf(d3.y, 0.8455960154533386f, bi);
    ar = fmaf(s4.x, -0.956400990486145f, ar); ai = fmaf(s4.y, -0.956400990486145f, ai); br = fmaf(d4.x, 0.29205676913261414f, br); bi = fmaf(d4.y, 0.29205676913261414f, bi);
    ar = fmaf(s5.x, -0.9151456356048584f, ar); ai = fmaf(s5.y, -0.9151456356048584f, ai); br = fmaf(d5.x, -0.4031234383583069f, br); bi = fmaf(d5.y, -0.4031234383583069f, bi);
    ar = fmaf(s6.x, -0.43006521463394165f, ar); ai = fmaf(s6.y, -0.43006521463394165f, ai); br = fmaf(d6.x, -0.9027978181838989f, br); bi = fmaf(d6.y, -0.9027978181838989f, bi);
    ar = fmaf(s7.x, 0.26358717679977417f, ar); ai = fmaf(s7.y, 0.26358717679977417f, ai); br = fmaf(d7.x, -0.9646356105804443f, br); bi = fmaf(d7.y, -0.9646356105804443f, bi);
    ar = fmaf(s8.x, 0.829405665397644f, ar); ai = fmaf(s8.y, 0.829405665397644f, ai); br = fmaf(d8.x, -0.5586467385292053f, br); bi = fmaf(d8.y, -0.5586467385292053f, bi);
    ar = fmaf(s9.x, 0.9929810762405396f, ar); ai = fmaf(s9.y, 0.9929810762405396f, ai); br = fmaf(d9.x, 0.11827316880226135f, br); bi = fmaf(d9.y, 0.11827316880226135f, bi);
    ar = fmaf(s10.x, 0.674983024597168f, ar); ai = fmaf(s10.y, 0.674983024597168f, ai); br = fmaf(d10.x, 0.7378332614898682f, br); bi = fmaf(d10.y, 0.7378332614898682f, bi);
    ar = fmaf(s11.x, 0.029633328318595886f, ar); ai = fmaf(s11.y, 0.029633328318595886f, ai); br = fmaf(d11.x, 0.9995608329772949f, br); bi = fmaf(d11.y, 0.9995608329772949f, bi);
    ar = fmaf(s12.x, -0.6300878524780273f, ar); ai = fmaf(s12.y, -0.6300878524780273f, ai); br = fmaf(d12.x, 0.7765238881111145f, br); bi = fmaf(d12.y, 0.7765238881111145f, bi);
    ar = fmaf(s13.x, -0.9842305779457092f, ar); ai = fmaf(s13.y, -0.9842305779457092f, ai); br = fmaf(d13.x, 0.1768902689218521f, br); bi = fmaf(d13.y, 0.1768902689218521f, bi);
    ar = fmaf(s14.x, -0.8610436320304871f, ar); ai = fmaf(s14.y, -0.8610436320304871f, ai); br = fmaf(d14.x, -0.5085310935974121f, br); bi = fmaf(d14.y, -0.5085310935974121f, bi);
    ar = fmaf(s15.x, -0.3202698528766632f, ar); ai = fmaf(s15.y, -0.3202698528766632f, ai); br = fmaf(d15.x, -0.9473263621330261f, br); bi = fmaf(d15.y, -0.9473263621330261f, bi);
    ar = fmaf(s16.x, 0.3758275806903839f, ar); ai = fmaf(s16.y, 0.3758275806903839f, ai); br = fmaf(d16.x, -0.926689624786377f, br); bi = fmaf(d16.y, -0.926689624786377f, bi);
    ar = fmaf(s17.x, 0.8896570801734924f, ar); ai = fmaf(s17.y, 0.8896570801734924f, ai); br = fmaf(d17.x, -0.4566292464733124f, br); bi = fmaf(d17.y, -0.4566292464733124f, bi);
    ar = fmaf(s18.x, 0.9720228910446167f, ar); ai = fmaf(s18.y, 0.9720228910446167f, ai); br = fmaf(d18.x, 0.2348860502243042f, br); bi = fmaf(d18.y, 0.2348860502243042f, bi);
    ar = fmaf(s19.x, 0.5829795002937317f, ar); ai = fmaf(s19.y, 0.5829795002937317f, ai); br = fmaf(d19.x, 0.8124868869781494f, br); bi = fmaf(d19.y, 0.8124868869781494f, bi);
    ar = fmaf(s20.x, -0.08879589289426804f, ar); ai = fmaf(s20.y, -0.08879589289426804f, ai); br = fmaf(d20.x, 0.9960498213768005f, br); bi = fmaf(d20.y, 0.9960498213768005f, bi);
    ar = fmaf(s21.x, -0.7175072431564331f, ar); ai = fmaf(s21.y, -0.7175072431564331f, ai); br = fmaf(d21.x, 0.6965510249137878f, br); bi = fmaf(d21.y, 0.6965510249137878f, bi);
    ar = fmaf(s22.x, -0.9982437491416931f, ar); ai = fmaf(s22.y, -0.9982437491416931f, ai); br = fmaf(d22.x, 0.05924062803387642f, br); bi = fmaf(d22.y, 0.05924062803387642f, bi);
    ar = fmaf(s23.x, -0.794854462146759f, ar); ai = fmaf(s23.y, -0.794854462146759f, ai); br = fmaf(d23.x, -0.6068001389503479f, br); bi = fmaf(d23.y, -0.6068001389503479f, bi);
    ar = fmaf(s24.x, -0.2059786170721054f, ar); ai = fmaf(s24.y, -0.2059786170721054f, ai); br = fmaf(d24.x, -0.9785565137863159f, br); bi = fmaf(d24.y, -0.9785565137863159f, bi);
    ar = fmaf(s25.x, 0.4827921986579895f, ar); ai = fmaf(s25.y, 0.4827921986579895f, ai); br = fmaf(d25.x, -0.8757349252700806f, br); bi = fmaf(d25.y, -0.8757349252700806f, bi);
    ar = fmaf(s26.x, 0.9374196529388428f, ar); ai = fmaf(s26.y, 0.9374196529388428f, ai); br = fmaf(d26.x, -0.3482016324996948f, br); bi = fmaf(d26.y, -0.3482016324996948f, bi);
    if (!INV) {
      v[6] = make_float2(ar + bi, ai - br); v[47] = make_float2(ar - bi, ai + br);
    } else {
      v[6] = make_float2(ar - bi, ai + br); v[47] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.674983024597168f, ar); ai = fmaf(s1.y, 0.674983024597168f, ai); br = fmaf(d1.x, 0.7378332614898682f, br); bi = fmaf(d1.y, 0.7378332614898682f, bi);
    ar = fmaf(s2.x, -0.08879589289426804f, ar); ai = fmaf(s2.y, -0.08879589289426804f, ai); br = fmaf(d2.x, 0.9960498213768005f, br); bi = fmaf(d2.y, 0.9960498213768005f, bi);
    ar = fmaf(s3.x, -0.794854462146759f, ar); ai = fmaf(s3.y, -0.794854462146759f, ai); br = fmaf(d3.x, 0.6068001389503479f, br); bi = fmaf(d3.y, 0.6068001389503479f, bi);
    ar = fmaf(s4.x, -0.9842305779457092f, ar); ai = fmaf(s4.y, -0.9842305779457092f, ai); br = fmaf(d4.x, -0.1768902689218521f, br); bi = fmaf(d4.y, -0.1768902689218521f, bi);
    ar = fmaf(s5.x, -0.5338233709335327f, ar); ai = fmaf(s5.y, -0.5338233709335327f, ai); br = fmaf(d5.x, -0.8455960154533386f, br); bi = fmaf(d5.y, -0.8455960154533386f, bi);
    ar = fmaf(s6.x, 0.26358717679977417f, ar); ai = fmaf(s6.y, 0.26358717679977417f, ai); br = fmaf(d6.x, -0.9646356105804443f, br); bi = fmaf(d6.y, -0.9646356105804443f, bi);
    ar = fmaf(s7.x, 0.8896570801734924f, ar); ai = fmaf(s7.y, 0.8896570801734924f, ai); br = fmaf(d7.x, -0.4566292464733124f, br); bi = fmaf(d7.y, -0.4566292464733124f, bi);
    ar = fmaf(s8.x, 0.9374196529388428f, ar); ai = fmaf(s8.y, 0.9374196529388428f, ai); br = fmaf(d8.x, 0.3482016324996948f, br); bi = fmaf(d8.y, 0.3482016324996948f, bi);
    ar = fmaf(s9.x, 0.3758275806903839f, ar); ai = fmaf(s9.y, 0.3758275806903839f, ai); br = fmaf(d9.x, 0.926689624786377f, br); bi = fmaf(d9.y, 0.926689624786377f, bi);
    ar = fmaf(s10.x, -0.43006521463394165f, ar); ai = fmaf(s10.y, -0.43006521463394165f, ai); br = fmaf(d10.x, 0.9027978181838989f, br); bi = fmaf(d10.y, 0.9027978181838989f, bi);
    ar = fmaf(s11.x, -0.956400990486145f, ar); ai = fmaf(s11.y, -0.956400990486145f, ai); br = fmaf(d11.x, 0.29205676913261414f, br); bi = fmaf(d11.y, 0.29205676913261414f, bi);
    ar = fmaf(s12.x, -0.8610436320304871f, ar); ai = fmaf(s12.y, -0.8610436320304871f, ai); br = fmaf(d12.x, -0.5085310935974121f, br); bi = fmaf(d12.y, -0.5085310935974121f, bi);
    ar = fmaf(s13.x, -0.2059786170721054f, ar); ai = fmaf(s13.y, -0.2059786170721054f, ai); br = fmaf(d13.x, -0.9785565137863159f, br); bi = fmaf(d13.y, -0.9785565137863159f, bi);
    ar = fmaf(s14.x, 0.5829795002937317f, ar); ai = fmaf(s14.y, 0.5829795002937317f, ai); br = fmaf(d14.x, -0.8124868869781494f, br); bi = fmaf(d14.y, -0.8124868869781494f, bi);
    ar = fmaf(s15.x, 0.9929810762405396f, ar); ai = fmaf(s15.y, 0.9929810762405396f, ai); br = fmaf(d15.x, -0.11827316880226135f, br); bi = fmaf(d15.y, -0.11827316880226135f, bi);
    ar = fmaf(s16.x, 0.7575112581253052f, ar); ai = fmaf(s16.y, 0.7575112581253052f, ai); br = fmaf(d16.x, 0.6528221368789673f, br); bi = fmaf(d16.y, 0.6528221368789673f, bi);
    ar = fmaf(s17.x, 0.029633328318595886f, ar); ai = fmaf(s17.y, 0.029633328318595886f, ai); br = fmaf(d17.x, 0.9995608329772949f, br); bi = fmaf(d17.y, 0.9995608329772949f, bi);
    ar = fmaf(s18.x, -0.7175072431564331f, ar); ai = fmaf(s18.y, -0.7175072431564331f, ai); br = fmaf(d18.x, 0.6965510249137878f, br); bi = fmaf(d18.y, 0.6965510249137878f, bi);
    ar = fmaf(s19.x, -0.9982437491416931f, ar); ai = fmaf(s19.y, -0.9982437491416931f, ai); br = fmaf(d19.x, -0.05924062803387642f, br); bi = fmaf(d19.y, -0.05924062803387642f, bi);
    ar = fmaf(s20.x, -0.6300878524780273f, ar); ai = fmaf(s20.y, -0.6300878524780273f, ai); br = fmaf(d20.x, -0.7765238881111145f, br); bi = fmaf(d20.y, -0.7765238881111145f, bi);
    ar = fmaf(s21.x, 0.14764656126499176f, ar); ai = fmaf(s21.y, 0.14764656126499176f, ai); br = fmaf(d21.x, -0.989040195941925f, br); bi = fmaf(d21.y, -0.989040195941925f, bi);
    ar = fmaf(s22.x, 0.829405665397644f, ar); ai = fmaf(s22.y, 0.829405665397644f, ai); br = fmaf(d22.x, -0.5586467385292053f, br); bi = fmaf(d22.y, -0.5586467385292053f, bi);
    ar = fmaf(s23.x, 0.9720228910446167f, ar); ai = fmaf(s23.y, 0.9720228910446167f, ai); br = fmaf(d23.x, 0.2348860502243042f, br); bi = fmaf(d23.y, 0.2348860502243042f, bi);
    ar = fmaf(s24.x, 0.4827921986579895f, ar); ai = fmaf(s24.y, 0.4827921986579895f, ai); br = fmaf(d24.x, 0.8757349252700806f, br); bi = fmaf(d24.y, 0.8757349252700806f, bi);
    ar = fmaf(s25.x, -0.3202698528766632f, ar); ai = fmaf(s25.y, -0.3202698528766632f, ai); br = fmaf(d25.x, 0.9473263621330261f, br); bi = fmaf(d25.y, 0.9473263621330261f, bi);
    ar = fmaf(s26.x, -0.9151456356048584f, ar); ai = fmaf(s26.y, -0.9151456356048584f, ai); br = fmaf(d26.x, 0.4031234383583069f, br); bi = fmaf(d26.y, 0.4031234383583069f, bi);
    if (!INV) {
      v[7] = make_float2(ar + bi, ai - br); v[46] = make_float2(ar - bi, ai + br);
    } else {
      v[7] = make_float2(ar - bi, ai + br); v[46] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.5829795002937317f, ar); ai = fmaf(s1.y, 0.5829795002937317f, ai); br = fmaf(d1.x, 0.8124868869781494f, br); bi = fmaf(d1.y, 0.8124868869781494f, bi);
    ar = fmaf(s2.x, -0.3202698528766632f, ar); ai = fmaf(s2.y, -0.3202698528766632f, ai); br = fmaf(d2.x, 0.9473263621330261f, br); bi = fmaf(d2.y, 0.9473263621330261f, bi);
    ar = fmaf(s3.x, -0.956400990486145f, ar); ai = fmaf(s3.y, -0.956400990486145f, ai); br = fmaf(d3.x, 0.29205676913261414f, br); bi = fmaf(d3.y, 0.29205676913261414f, bi);
    ar = fmaf(s4.x, -0.794854462146759f, ar); ai = fmaf(s4.y, -0.794854462146759f, ai); br = fmaf(d4.x, -0.6068001389503479f, br); bi = fmaf(d4.y, -0.6068001389503479f, bi);
    ar = fmaf(s5.x, 0.029633328318595886f, ar); ai = fmaf(s5.y, 0.029633328318595886f, ai); br = fmaf(d5.x, -0.9995608329772949f, br); bi = fmaf(d5.y, -0.9995608329772949f, bi);
    ar = fmaf(s6.x, 0.829405665397644f, ar); ai = fmaf(s6.y, 0.829405665397644f, ai); br = fmaf(d6.x, -0.5586467385292053f, br); bi = fmaf(d6.y, -0.5586467385292053f, bi);
    ar = fmaf(s7.x, 0.9374196529388428f, ar); ai = fmaf(s7.y, 0.9374196529388428f, ai); br = fmaf(d7.x, 0.3482016324996948f, br); bi = fmaf(d7.y, 0.3482016324996948f, bi);
    ar = fmaf(s8.x, 0.26358717679977417f, ar); ai = fmaf(s8.y, 0.26358717679977417f, ai); br = fmaf(d8.x, 0.9646356105804443f, br); bi = fmaf(d8.y, 0.9646356105804443f, bi);
    ar = fmaf(s9.x, -0.6300878524780273f, ar); ai = fmaf(s9.y, -0.6300878524780273f, ai); br = fmaf(d9.x, 0.7765238881111145f, br); bi = fmaf(d9.y, 0.7765238881111145f, bi);
    ar = fmaf(s10.x, -0.9982437491416931f, ar); ai = fmaf(s10.y, -0.9982437491416931f, ai); br = fmaf(d10.x, -0.05924062803387642f, br); bi = fmaf(d10.y, -0.05924062803387642f, bi);
    ar = fmaf(s11.x, -0.5338233709335327f, ar); ai = fmaf(s11.y, -0.5338233709335327f, ai); br = fmaf(d11.x, -0.8455960154533386f, br); bi = fmaf(d11.y, -0.8455960154533386f, bi);
    ar = fmaf(s12.x, 0.3758275806903839f, ar); ai = fmaf(s12.y, 0.3758275806903839f, ai); br = fmaf(d12.x, -0.926689624786377f, br); bi = fmaf(d12.y, -0.926689624786377f, bi);
    ar = fmaf(s13.x, 0.9720228910446167f, ar); ai = fmaf(s13.y, 0.9720228910446167f, ai); br = fmaf(d13.x, -0.2348860502243042f, br); bi = fmaf(d13.y, -0.2348860502243042f, bi);
    ar = fmaf(s14.x, 0.7575112581253052f, ar); ai = fmaf(s14.y, 0.7575112581253052f, ai); br = fmaf(d14.x, 0.6528221368789673f, br); bi = fmaf(d14.y, 0.6528221368789673f, bi);
    ar = fmaf(s15.x, -0.08879589289426804f, ar); ai = fmaf(s15.y, -0.08879589289426804f, ai); br = fmaf(d15.x, 0.9960498213768005f, br); bi = fmaf(d15.y, 0.9960498213768005f, bi);
    ar = fmaf(s16.x, -0.8610436320304871f, ar); ai = fmaf(s16.y, -0.8610436320304871f, ai); br = fmaf(d16.x, 0.5085310935974121f, br); bi = fmaf(d16.y, 0.5085310935974121f, bi);
    ar = fmaf(s17.x, -0.9151456356048584f, ar); ai = fmaf(s17.y, -0.9151456356048584f, ai); br = fmaf(d17.x, -0.4031234383583069f, br); bi = fmaf(d17.y, -0.4031234383583069f, bi);
    ar = fmaf(s18.x, -0.2059786170721054f, ar); ai = fmaf(s18.y, -0.2059786170721054f, ai); br = fmaf(d18.x, -0.9785565137863159f, br); bi = fmaf(d18.y, -0.9785565137863159f, bi);
    ar = fmaf(s19.x, 0.674983024597168f, ar); ai = fmaf(s19.y, 0.674983024597168f, ai); br = fmaf(d19.x, -0.7378332614898682f, br); bi = fmaf(d19.y, -0.7378332614898682f, bi);
    ar = fmaf(s20.x, 0.9929810762405396f, ar); ai = fmaf(s20.y, 0.9929810762405396f, ai); br = fmaf(d20.x, 0.11827316880226135f, br); bi = fmaf(d20.y, 0.11827316880226135f, bi);
    ar = fmaf(s21.x, 0.4827921986579895f, ar); ai = fmaf(s21.y, 0.4827921986579895f, ai); br = fmaf(d21.x, 0.8757349252700806f, br); bi = fmaf(d21.y, 0.8757349252700806f, bi);
    ar = fmaf(s22.x, -0.43006521463394165f, ar); ai = fmaf(s22.y, -0.43006521463394165f, ai); br = fmaf(d22.x, 0.9027978181838989f, br); bi = fmaf(d22.y, 0.9027978181838989f, bi);
    ar = fmaf(s23.x, -0.9842305779457092f, ar); ai = fmaf(s23.y, -0.9842305779457092f, ai); br = fmaf(d23.x, 0.1768902689218521f, br); bi = fmaf(d23.y, 0.1768902689218521f, bi);
    ar = fmaf(s24.x, -0.7175072431564331f, ar); ai = fmaf(s24.y, -0.7175072431564331f, ai); br = fmaf(d24.x, -0.6965510249137878f, br); bi = fmaf(d24.y, -0.6965510249137878f, bi);
    ar = fmaf(s25.x, 0.14764656126499176f, ar); ai = fmaf(s25.y, 0.14764656126499176f, ai); br = fmaf(d25.x, -0.989040195941925f, br); bi = fmaf(d25.y, -0.989040195941925f, bi);
    ar = fmaf(s26.x, 0.8896570801734924f, ar); ai = fmaf(s26.y, 0.8896570801734924f, ai); br = fmaf(d26.x, -0.4566292464733124f, br); bi = fmaf(d26.y, -0.4566292464733124f, bi);
    if (!INV) {
      v[8] = make_float2(ar + bi, ai - br); v[45] = make_float2(ar - bi, ai + br);
    } else {
      v[8] = make_float2(ar - bi, ai + br); v[45] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.4827921986579895f, ar); ai = fmaf(s1.y, 0.4827921986579895f, ai); br = fmaf(d1.x, 0.8757349252700806f, br); bi = fmaf(d1.y, 0.8757349252700806f, bi);
    ar = fmaf(s2.x, -0.5338233709335327f, ar); ai = fmaf(s2.y, -0.5338233709335327f, ai); br = fmaf(d2.x, 0.8455960154533386f, br); bi = fmaf(d2.y, 0.8455960154533386f, bi);
    ar = fmaf(s3.x, -0.9982437491416931f, ar); ai = fmaf(s3.y, -0.9982437491416931f, ai); br = fmaf(d3.x, -0.05924062803387642f, br); bi = fmaf(d3.y, -0.05924062803387642f, bi);
    ar = fmaf(s4.x, -0.43006521463394165f, ar); ai = fmaf(s4.y, -0.43006521463394165f, ai); br = fmaf(d4.x, -0.9027978181838989f, br); bi = fmaf(d4.y, -0.9027978181838989f, bi);
    ar = fmaf(s5.x, 0.5829795002937317f, ar); ai = fmaf(s5.y, 0.5829795002937317f, ai); br = fmaf(d5.x, -0.8124868869781494f, br); bi = fmaf(d5.y, -0.8124868869781494f, bi);
    ar = fmaf(s6.x, 0.9929810762405396f, ar); ai = fmaf(s6.y, 0.9929810762405396f, ai); br = fmaf(d6.x, 0.11827316880226135f, br); bi = fmaf(d6.y, 0.11827316880226135f, bi);
    ar = fmaf(s7.x, 0.3758275806903839f, ar); ai = fmaf(s7.y, 0.3758275806903839f, ai); br = fmaf(d7.x, 0.926689624786377f, br); bi = fmaf(d7.y, 0.926689624786377f, bi);
    ar = fmaf(s8.x, -0.6300878524780273f, ar); ai = fmaf(s8.y, -0.6300878524780273f, ai); br = fmaf(d8.x, 0.7765238881111145f, br); bi = fmaf(d8.y, 0.7765238881111145f, bi);
    ar = fmaf(s9.x, -0.9842305779457092f, ar); ai = fmaf(s9.y, -0.9842305779457092f, ai); br = fmaf(d9.x, -0.1768902689218521f, br); bi = fmaf(d9.y, -0.1768902689218521f, bi);
    ar = fmaf(s10.x, -0.3202698528766632f, ar); ai = fmaf(s10.y, -0.3202698528766632f, ai); br = fmaf(d10.x, -0.9473263621330261f, br); bi = fmaf(d10.y, -0.9473263621330261f, bi);
    ar = fmaf(s11.x, 0.674983024597168f, ar); ai = fmaf(s11.y, 0.674983024597168f, ai); br = fmaf(d11.x, -0.7378332614898682f, br); bi = fmaf(d11.y, -0.7378332614898682f, bi);
    ar = fmaf(s12.x, 0.9720228910446167f, ar); ai = fmaf(s12.y, 0.9720228910446167f, ai); br = fmaf(d12.x, 0.2348860502243042f, br); bi = fmaf(d12.y, 0.2348860502243042f, bi);
    ar = fmaf(s13.x, 0.26358717679977417f, ar); ai = fmaf(s13.y, 0.26358717679977417f, ai); br = fmaf(d13.x, 0.9646356105804443f, br); bi = fmaf(d13.y, 0.9646356105804443f, bi);
    ar = fmaf(s14.x, -0.7175072431564331f, ar); ai = fmaf(s14.y, -0.7175072431564331f, ai); br = fmaf(d14.x, 0.6965510249137878f, br); bi = fmaf(d14.y, 0.6965510249137878f, bi);
    ar = fmaf(s15.x, -0.956400990486145f, ar); ai = fmaf(s15.y, -0.956400990486145f, ai); br = fmaf(d15.x, -0.29205676913261414f, br); bi = fmaf(d15.y, -0.29205676913261414f, bi);
    ar = fmaf(s16.x, -0.2059786170721054f, ar); ai = fmaf(s16.y, -0.2059786170721054f, ai); br = fmaf(d16.x, -0.9785565137863159f, br); bi = fmaf(d16.y, -0.9785565137863159f, bi);
    ar = fmaf(s17.x, 0.7575112581253052f, ar); ai = fmaf(s17.y, 0.7575112581253052f, ai); br = fmaf(d17.x, -0.6528221368789673f, br); bi = fmaf(d17.y, -0.6528221368789673f, bi);
    ar = fmaf(s18.x, 0.9374196529388428f, ar); ai = fmaf(s18.y, 0.9374196529388428f, ai); br = fmaf(d18.x, 0.3482016324996948f, br); bi = fmaf(d18.y, 0.3482016324996948f, bi);
    ar = fmaf(s19.x, 0.14764656126499176f, ar); ai = fmaf(s19.y, 0.14764656126499176f, ai); br = fmaf(d19.x, 0.989040195941925f, br); bi = fmaf(d19.y, 0.989040195941925f, bi);
    ar = fmaf(s20.x, -0.794854462146759f, ar); ai = fmaf(s20.y, -0.794854462146759f, ai); br = fmaf(d20.x, 0.6068001389503479f, br); bi = fmaf(d20.y, 0.6068001389503479f, bi);
    ar = fmaf(s21.x, -0.9151456356048584f, ar); ai = fmaf(s21.y, -0.9151456356048584f, ai); br = fmaf(d21.x, -0.4031234383583069f, br); bi = fmaf(d21.y, -0.4031234383583069f, bi);
    ar = fmaf(s22.x, -0.08879589289426804f, ar); ai = fmaf(s22.y, -0.08879589289426804f, ai); br = fmaf(d22.x, -0.9960498213768005f, br); bi = fmaf(d22.y, -0.9960498213768005f, bi);
    ar = fmaf(s23.x, 0.829405665397644f, ar); ai = fmaf(s23.y, 0.829405665397644f, ai); br = fmaf(d23.x, -0.5586467385292053f, br); bi = fmaf(d23.y, -0.5586467385292053f, bi);
    ar = fmaf(s24.x, 0.8896570801734924f, ar); ai = fmaf(s24.y, 0.8896570801734924f, ai); br = fmaf(d24.x, 0.4566292464733124f, br); bi = fmaf(d24.y, 0.4566292464733124f, bi);
    ar = fmaf(s25.x, 0.029633328318595886f, ar); ai = fmaf(s25.y, 0.029633328318595886f, ai); br = fmaf(d25.x, 0.9995608329772949f, br); bi = fmaf(d25.y, 0.9995608329772949f, bi);
    ar = fmaf(s26.x, -0.8610436320304871f, ar); ai = fmaf(s26.y, -0.8610436320304871f, ai); br = fmaf(d26.x, 0.5085310935974121f, br); bi = fmaf(d26.y, 0.5085310935974121f, bi);
    if (!INV) {
      v[9] = make_float2(ar + bi, ai - br); v[44] = make_float2(ar - bi, ai + br);
    } else {
      v[9] = make_float2(ar - bi, ai + br); v[44] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.3758275806903839f, ar); ai = fmaf(s1.y, 0.3758275806903839f, ai); br = fmaf(d1.x, 0.926689624786377f, br); bi = fmaf(d1.y, 0.926689624786377f, bi);
    ar = fmaf(s2.x, -0.7175072431564331f, ar); ai = fmaf(s2.y, -0.7175072431564331f, ai); br = fmaf(d2.x, 0.6965510249137878f, br); bi = fmaf(d2.y, 0.6965510249137878f, bi);
    ar = fmaf(s3.x, -0.9151456356048584f, ar); ai = fmaf(s3.y, -0.9151456356048584f, ai); br = fmaf(d3.x, -0.4031234383583069f, br); bi = fmaf(d3.y, -0.4031234383583069f, bi);
    ar = fmaf(s4.x, 0.029633328318595886f, ar); ai = fmaf(s4.y, 0.029633328318595886f, ai); br = fmaf(d4.x, -0.9995608329772949f, br); bi = fmaf(d4.y, -0.9995608329772949f, bi);
    ar = fmaf(s5.x, 0.9374196529388428f, ar); ai = fmaf(s5.y, 0.9374196529388428f, ai); br = fmaf(d5.x, -0.3482016324996948f, br); bi = fmaf(d5.y, -0.3482016324996948f, bi);
    ar = fmaf(s6.x, 0.674983024597168f, ar); ai = fmaf(s6.y, 0.674983024597168f, ai); br = fmaf(d6.x, 0.7378332614898682f, br); bi = fmaf(d6.y, 0.7378332614898682f, bi);
    ar = fmaf(s7.x, -0.43006521463394165f, ar); ai = fmaf(s7.y, -0.43006521463394165f, ai); br = fmaf(d7.x, 0.9027978181838989f, br); bi = fmaf(d7.y, 0.9027978181838989f, bi);
    ar = fmaf(s8.x, -0.9982437491416931f, ar); ai = fmaf(s8.y, -0.9982437491416931f, ai); br = fmaf(d8.x, -0.05924062803387642f, br); bi = fmaf(d8.y, -0.05924062803387642f, bi);
    ar = fmaf(s9.x, -0.3202698528766632f, ar); ai = fmaf(s9.y, -0.3202698528766632f, ai); br = fmaf(d9.x, -0.9473263621330261f, br); bi = fmaf(d9.y, -0.9473263621330261f, bi);
    ar = fmaf(s10.x, 0.7575112581253052f, ar); ai = fmaf(s10.y, 0.7575112581253052f, ai); br = fmaf(d10.x, -0.6528221368789673f, br); bi = fmaf(d10.y, -0.6528221368789673f, bi);
    ar = fmaf(s11.x, 0.8896570801734924f, ar); ai = fmaf(s11.y, 0.8896570801734924f, ai); br = fmaf(d11.x, 0.4566292464733124f, br); bi = fmaf(d11.y, 0.4566292464733124f, bi);
    ar = fmaf(s12.x, -0.08879589289426804f, ar); ai = fmaf(s12.y, -0.08879589289426804f, ai); br = fmaf(d12.x, 0.9960498213768005f, br); bi = fmaf(d12.y, 0.9960498213768005f, bi);
    ar = fmaf(s13.x, -0.956400990486145f, ar); ai = fmaf(s13.y, -0.956400990486145f, ai); br = fmaf(d13.x, 0.29205676913261414f, br); bi = fmaf(d13.y, 0.29205676913261414f, bi);
    ar = fmaf(s14.x, -0.6300878524780273f, ar); ai = fmaf(s14.y, -0.6300878524780273f, ai); br = fmaf(d14.x, -0.7765238881111145f, br); bi = fmaf(d14.y, -0.7765238881111145f, bi);
    ar = fmaf(s15.x, 0.4827921986579895f, ar); ai = fmaf(s15.y, 0.4827921986579895f, ai); br = fmaf(d15.x, -0.8757349252700806f, br); bi = fmaf(d15.y, -0.8757349252700806f, bi);
    ar = fmaf(s16.x, 0.9929810762405396f, ar); ai = fmaf(s16.y, 0.9929810762405396f, ai); br = fmaf(d16.x, 0.11827316880226135f, br); bi = fmaf(d16.y, 0.11827316880226135f, bi);
    ar = fmaf(s17.x, 0.26358717679977417f, ar); ai = fmaf(s17.y, 0.26358717679977417f, ai); br = fmaf(d17.x, 0.9646356105804443f, br); bi = fmaf(d17.y, 0.9646356105804443f, bi);
    ar = fmaf(s18.x, -0.794854462146759f, ar); ai = fmaf(s18.y, -0.794854462146759f, ai); br = fmaf(d18.x, 0.6068001389503479f, br); bi = fmaf(d18.y, 0.6068001389503479f, bi);
    ar = fmaf(s19.x, -0.8610436320304871f, ar); ai = fmaf(s19.y, -0.8610436320304871f, ai); br = fmaf(d19.x, -0.5085310935974121f, br); bi = fmaf(d19.y, -0.5085310935974121f, bi);
    ar = fmaf(s20.x, 0.14764656126499176f, ar); ai = fmaf(s20.y, 0.14764656126499176f, ai); br = fmaf(d20.x, -0.989040195941925f, br); bi = fmaf(d20.y, -0.989040195941925f, bi);
    ar = fmaf(s21.x, 0.9720228910446167f, ar); ai = fmaf(s21.y, 0.9720228910446167f, ai); br = fmaf(d21.x, -0.2348860502243042f, br); bi = fmaf(d21.y, -0.2348860502243042f, bi);
    ar = fmaf(s22.x, 0.5829795002937317f, ar); ai = fmaf(s22.y, 0.5829795002937317f, ai); br = fmaf(d22.x, 0.8124868869781494f, br); bi = fmaf(d22.y, 0.8124868869781494f, bi);
    ar = fmaf(s23.x, -0.5338233709335327f, ar); ai = fmaf(s23.y, -0.5338233709335327f, ai); br = fmaf(d23.x, 0.8455960154533386f, br); bi = fmaf(d23.y, 0.8455960154533386f, bi);
    ar = fmaf(s24.x, -0.9842305779457092f, ar); ai = fmaf(s24.y, -0.9842305779457092f, ai); br = fmaf(d24.x, -0.1768902689218521f, br); bi = fmaf(d24.y, -0.1768902689218521f, bi);
    ar = fmaf(s25.x, -0.2059786170721054f, ar); ai = fmaf(s25.y, -0.2059786170721054f, ai); br = fmaf(d25.x, -0.9785565137863159f, br); bi = fmaf(d25.y, -0.9785565137863159f, bi);
    ar = fmaf(s26.x, 0.829405665397644f, ar); ai = fmaf(s26.y, 0.829405665397644f, ai); br = fmaf(d26.x, -0.5586467385292053f, br); bi = fmaf(d26.y, -0.5586467385292053f, bi);
    if (!INV) {
      v[10] = make_float2(ar + bi, ai - br); v[43] = make_float2(ar - bi, ai + br);
    } else {
      v[10] = make_float2(ar - bi, ai + br); v[43] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.26358717679977417f, ar); ai = fmaf(s1.y, 0.26358717679977417f, ai); br = fmaf(d1.x, 0.9646356105804443f, br); bi = fmaf(d1.y, 0.9646356105804443f, bi);
    ar = fmaf(s2.x, -0.8610436320304871f, ar); ai = fmaf(s2.y, -0.8610436320304871f, ai); br = fmaf(d2.x, 0.5085310935974121f, br); bi = fmaf(d2.y, 0.5085310935974121f, bi);
    ar = fmaf(s3.x, -0.7175072431564331f, ar); ai = fmaf(s3.y, -0.7175072431564331f, ai); br = fmaf(d3.x, -0.6965510249137878f, br); bi = fmaf(d3.y, -0.6965510249137878f, bi);
    ar = fmaf(s4.x, 0.4827921986579895f, ar); ai = fmaf(s4.y, 0.4827921986579895f, ai); br = fmaf(d4.x, -0.8757349252700806f, br); bi = fmaf(d4.y, -0.8757349252700806f, bi);
    ar = fmaf(s5.x, 0.9720228910446167f, ar); ai = fmaf(s5.y, 0.9720228910446167f, ai); br = fmaf(d5.x, 0.2348860502243042f, br); bi = fmaf(d5.y, 0.2348860502243042f, bi);
    ar = fmaf(s6.x, 0.029633328318595886f, ar); ai = fmaf(s6.y, 0.029633328318595886f, ai); br = fmaf(d6.x, 0.9995608329772949f, br); bi = fmaf(d6.y, 0.9995608329772949f, bi);
    ar = fmaf(s7.x, -0.956400990486145f, ar); ai = fmaf(s7.y, -0.956400990486145f, ai); br = fmaf(d7.x, 0.29205676913261414f, br); bi = fmaf(d7.y, 0.29205676913261414f, bi);
    ar = fmaf(s8.x, -0.5338233709335327f, ar); ai = fmaf(s8.y, -0.5338233709335327f, ai); br = fmaf(d8.x, -0.8455960154533386f, br); bi = fmaf(d8.y, -0.8455960154533386f, bi);
    ar = fmaf(s9.x, 0.674983024597168f, ar); ai = fmaf(s9.y, 0.674983024597168f, ai); br = fmaf(d9.x, -0.7378332614898682f, br); bi = fmaf(d9.y, -0.7378332614898682f, bi);
    ar = fmaf(s10.x, 0.8896570801734924f, ar); ai = fmaf(s10.y, 0.8896570801734924f, ai); br = fmaf(d10.x, 0.4566292464733124f, br); bi = fmaf(d10.y, 0.4566292464733124f, bi);
    ar = fmaf(s11.x, -0.2059786170721054f, ar); ai = fmaf(s11.y, -0.2059786170721054f, ai); br = fmaf(d11.x, 0.9785565137863159f, br); bi = fmaf(d11.y, 0.9785565137863159f, bi);
    ar = fmaf(s12.x, -0.9982437491416931f, ar); ai = fmaf(s12.y, -0.9982437491416931f, ai); br = fmaf(d12.x, 0.05924062803387642f, br); bi = fmaf(d12.y, 0.05924062803387642f, bi);
    ar = fmaf(s13.x, -0.3202698528766632f, ar); ai = fmaf(s13.y, -0.3202698528766632f, ai); br = fmaf(d13.x, -0.9473263621330261f, br); bi = fmaf(d13.y, -0.9473263621330261f, bi);
    ar = fmaf(s14.x, 0.829405665397644f, ar); ai = fmaf(s14.y, 0.829405665397644f, ai); br = fmaf(d14.x, -0.5586467385292053f, br); bi = fmaf(d14.y, -0.5586467385292053f, bi);
    ar = fmaf(s15.x, 0.7575112581253052f, ar); ai = fmaf(s15.y, 0.7575112581253052f, ai); br = fmaf(d15.x, 0.6528221368789673f, br); bi = fmaf(d15.y, 0.6528221368789673f, bi);
    ar = fmaf(s16.x, -0.43006521463394165f, ar); ai = fmaf(s16.y, -0.43006521463394165f, ai); br = fmaf(d16.x, 0.9027978181838989f, br); bi = fmaf(d16.y, 0.9027978181838989f, bi);
    ar = fmaf(s17.x, -0.9842305779457092f, ar); ai = fmaf(s17.y, -0.9842305779457092f, ai); br = fmaf(d17.x, -0.1768902689218521f, br); bi = fmaf(d17.y, -0.1768902689218521f, bi);
    ar = fmaf(s18.x, -0.08879589289426804f, ar); ai = fmaf(s18.y, -0.08879589289426804f, ai); br = fmaf(d18.x, -0.9960498213768005f, br); bi = fmaf(d18.y, -0.9960498213768005f, bi);
    ar = fmaf(s19.x, 0.9374196529388428f, ar); ai = fmaf(s19.y, 0.9374196529388428f, ai); br = fmaf(d19.x, -0.3482016324996948f, br); bi = fmaf(d19.y, -0.3482016324996948f, bi);
    ar = fmaf(s20.x, 0.5829795002937317f, ar); ai = fmaf(s20.y, 0.5829795002937317f, ai); br = fmaf(d20.x, 0.8124868869781494f, br); bi = fmaf(d20.y, 0.8124868869781494f, bi);
    ar = fmaf(s21.x, -0.6300878524780273f, ar); ai = fmaf(s21.y, -0.6300878524780273f, ai); br = fmaf(d21.x, 0.7765238881111145f, br); bi = fmaf(d21.y, 0.7765238881111145f, bi);
    ar = fmaf(s22.x, -0.9151456356048584f, ar); ai = fmaf(s22.y, -0.9151456356048584f, ai); br = fmaf(d22.x, -0.4031234383583069f, br); bi = fmaf(d22.y, -0.4031234383583069f, bi);
    ar = fmaf(s23.x, 0.14764656126499176f, ar); ai = fmaf(s23.y, 0.14764656126499176f, ai); br = fmaf(d23.x, -0.989040195941925f, br); bi = fmaf(d23.y, -0.989040195941925f, bi);
    ar = fmaf(s24.x, 0.9929810762405396f, ar); ai = fmaf(s24.y, 0.9929810762405396f, ai); br = fmaf(d24.x, -0.11827316880226135f, br); bi = fmaf(d24.y, -0.11827316880226135f, bi);
    ar = fmaf(s25.x, 0.3758275806903839f, ar); ai = fmaf(s25.y, 0.3758275806903839f, ai); br = fmaf(d25.x, 0.926689624786377f, br); bi = fmaf(d25.y, 0.926689624786377f, bi);
    ar = fmaf(s26.x, -0.794854462146759f, ar); ai = fmaf(s26.y, -0.794854462146759f, ai); br = fmaf(d26.x, 0.6068001389503479f, br); bi = fmaf(d26.y, 0.6068001389503479f, bi);
    if (!INV) {
      v[11] = make_float2(ar + bi, ai - br); v[42] = make_float2(ar - bi, ai + br);
    } else {
      v[11] = make_float2(ar - bi, ai + br); v[42] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.14764656126499176f, ar); ai = fmaf(s1.y, 0.14764656126499176f, ai); br = fmaf(d1.x, 0.989040195941925f, br); bi = fmaf(d1.y, 0.989040195941925f, bi);
    ar = fmaf(s2.x, -0.956400990486145f, ar); ai = fmaf(s2.y, -0.956400990486145f, ai); br = fmaf(d2.x, 0.29205676913261414f, br); bi = fmaf(d2.y, 0.29205676913261414f, bi);
    ar = fmaf(s3.x, -0.43006521463394165f, ar); ai = fmaf(s3.y, -0.43006521463394165f, ai); br = fmaf(d3.x, -0.9027978181838989f, br); bi = fmaf(d3.y, -0.9027978181838989f, bi);
    ar = fmaf(s4.x, 0.829405665397644f, ar); ai = fmaf(s4.y, 0.829405665397644f, ai); br = fmaf(d4.x, -0.5586467385292053f, br); bi = fmaf(d4.y, -0.5586467385292053f, bi);
    ar = fmaf(s5.x, 0.674983024597168f, ar); ai = fmaf(s5.y, 0.674983024597168f, ai); br = fmaf(d5.x, 0.7378332614898682f, br); bi = fmaf(d5.y, 0.7378332614898682f, bi);
    ar = fmaf(s6.x, -0.6300878524780273f, ar); ai = fmaf(s6.y, -0.6300878524780273f, ai); br = fmaf(d6.x, 0.7765238881111145f, br); bi = fmaf(d6.y, 0.7765238881111145f, bi);
    ar = fmaf(s7.x, -0.8610436320304871f, ar); ai = fmaf(s7.y, -0.8610436320304871f, ai); br = fmaf(d7.x, -0.5085310935974121f, br); bi = fmaf(d7.y, -0.5085310935974121f, bi);
    ar = fmaf(s8.x, 0.3758275806903839f, ar); ai = fmaf(s8.y, 0.3758275806903839f, ai); br = fmaf(d8.x, -0.926689624786377f, br); bi = fmaf(d8.y, -0.926689624786377f, bi);
    ar = fmaf(s9.x, 0.9720228910446167f, ar); ai = fmaf(s9.y, 0.9720228910446167f, ai); br = fmaf(d9.x, 0.2348860502243042f, br); bi = fmaf(d9.y, 0.2348860502243042f, bi);
    ar = fmaf(s10.x, -0.08879589289426804f, ar); ai = fmaf(s10.y, -0.08879589289426804f, ai); br = fmaf(d10.x, 0.9960498213768005f, br); bi = fmaf(d10.y, 0.9960498213768005f, bi);
    ar = fmaf(s11.x, -0.9982437491416931f, ar); ai = fmaf(s11.y, -0.9982437491416931f, ai); br = fmaf(d11.x, 0.05924062803387642f, br); bi = fmaf(d11.y, 0.05924062803387642f, bi);
    ar = fmaf(s12.x, -0.2059786170721054f, ar); ai = fmaf(s12.y, -0.2059786170721054f, ai); br = fmaf(d12.x, -0.9785565137863159f, br); bi = fmaf(d12.y, -0.9785565137863159f, bi);
    ar = fmaf(s13.x, 0.9374196529388428f, ar); ai = fmaf(s13.y, 0.9374196529388428f, ai); br = fmaf(d13.x, -0.3482016324996948f, br); bi = fmaf(d13.y, -0.3482016324996948f, bi);
    ar = fmaf(s14.x, 0.4827921986579895f, ar); ai = fmaf(s14.y, 0.4827921986579895f, ai); br = fmaf(d14.x, 0.8757349252700806f, br); bi = fmaf(d14.y, 0.8757349252700806f, bi);
    ar = fmaf(s15.x, -0.794854462146759f, ar); ai = fmaf(s15.y, -0.794854462146759f, ai); br = fmaf(d15.x, 0.6068001389503479f, br); bi = fmaf(d15.y, 0.6068001389503479f, bi);
    ar = fmaf(s16.x, -0.7175072431564331f, ar); ai = fmaf(s16.y, -0.7175072431564331f, ai); br = fmaf(d16.x, -0.6965510249137878f, br); bi = fmaf(d16.y, -0.6965510249137878f, bi);
    ar = fmaf(s17.x, 0.5829795002937317f, ar); ai = fmaf(s17.y, 0.5829795002937317f, ai); br = fmaf(d17.x, -0.8124868869781494f, br); bi = fmaf(d17.y, -0.8124868869781494f, bi);
    ar = fmaf(s18.x, 0.8896570801734924f, ar); ai = fmaf(s18.y, 0.8896570801734924f, ai); br = fmaf(d18.x, 0.4566292464733124f, br); bi = fmaf(d18.y, 0.4566292464733124f, bi);
    ar = fmaf(s19.x, -0.3202698528766632f, ar); ai = fmaf(s19.y, -0.3202698528766632f, ai); br = fmaf(d19.x, 0.9473263621330261f, br); bi = fmaf(d19.y, 0.9473263621330261f, bi);
    ar = fmaf(s20.x, -0.9842305779457092f, ar); ai = fmaf(s20.y, -0.9842305779457092f, ai); br = fmaf(d20.x, -0.1768902689218521f, br); bi = fmaf(d20.y, -0.1768902689218521f, bi);
    ar = fmaf(s21.x, 0.029633328318595886f, ar); ai = fmaf(s21.y, 0.029633328318595886f, ai); br = fmaf(d21.x, -0.9995608329772949f, br); bi = fmaf(d21.y, -0.9995608329772949f, bi);
    ar = fmaf(s22.x, 0.9929810762405396f, ar); ai = fmaf(s22.y, 0.9929810762405396f, ai); br = fmaf(d22.x, -0.11827316880226135f, br); bi = fmaf(d22.y, -0.11827316880226135f, bi);
    ar = fmaf(s23.x, 0.26358717679977417f, ar); ai = fmaf(s23.y, 0.26358717679977417f, ai); br = fmaf(d23.x, 0.9646356105804443f, br); bi = fmaf(d23.y, 0.9646356105804443f, bi);
    ar = fmaf(s24.x, -0.9151456356048584f, ar); ai = fmaf(s24.y, -0.9151456356048584f, ai); br = fmaf(d24.x, 0.4031234383583069f, br); bi = fmaf(d24.y, 0.4031234383583069f, bi);
    ar = fmaf(s25.x, -0.5338233709335327f, ar); ai = fmaf(s25.y, -0.5338233709335327f, ai); br = fmaf(d25.x, -0.8455960154533386f, br); bi = fmaf(d25.y, -0.8455960154533386f, bi);
    ar = fmaf(s26.x, 0.7575112581253052f, ar); ai = fmaf(s26.y, 0.7575112581253052f, ai); br = fmaf(d26.x, -0.6528221368789673f, br); bi = fmaf(d26.y, -0.6528221368789673f, bi);
    if (!INV) {
      v[12] = make_float2(ar + bi, ai - br); v[41] = make_float2(ar - bi, ai + br);
    } else {
      v[12] = make_float2(ar - bi, ai + br); v[41] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, 0.029633328318595886f, ar); ai = fmaf(s1.y, 0.029633328318595886f, ai); br = fmaf(d1.x, 0.9995608329772949f, br); bi = fmaf(d1.y, 0.9995608329772949f, bi);
    ar = fmaf(s2.x, -0.9982437491416931f, ar); ai = fmaf(s2.y, -0.9982437491416931f, ai); br = fmaf(d2.x, 0.05924062803387642f, br); bi = fmaf(d2.y, 0.05924062803387642f, bi);
    ar = fmaf(s3.x, -0.08879589289426804f, ar); ai = fmaf(s3.y, -0.08879589289426804f, ai); br = fmaf(d3.x, -0.9960498213768005f, br); bi = fmaf(d3.y, -0.9960498213768005f, bi);
    ar = fmaf(s4.x, 0.9929810762405396f, ar); ai = fmaf(s4.y, 0.9929810762405396f, ai); br = fmaf(d4.x, -0.11827316880226135f, br); bi = fmaf(d4.y, -0.11827316880226135f, bi);
    ar = fmaf(s5.x, 0.14764656126499176f, ar); ai = fmaf(s5.y, 0.14764656126499176f, ai); br = fmaf(d5.x, 0.989040195941925f, br); bi = fmaf(d5.y, 0.989040195941925f, bi);
    ar = fmaf(s6.x, -0.9842305779457092f, ar); ai = fmaf(s6.y, -0.9842305779457092f, ai); br = fmaf(d6.x, 0.1768902689218521f, br); bi = fmaf(d6.y, 0.1768902689218521f, bi);
    ar = fmaf(s7.x, -0.2059786170721054f, ar); ai = fmaf(s7.y, -0.2059786170721054f, ai); br = fmaf(d7.x, -0.9785565137863159f, br); bi = fmaf(d7.y, -0.9785565137863159f, bi);
    ar = fmaf(s8.x, 0.9720228910446167f, ar); ai = fmaf(s8.y, 0.9720228910446167f, ai); br = fmaf(d8.x, -0.2348860502243042f, br); bi = fmaf(d8.y, -0.2348860502243042f, bi);
    ar = fmaf(s9.x, 0.26358717679977417f, ar); ai = fmaf(s9.y, 0.26358717679977417f, ai); br = fmaf(d9.x, 0.9646356105804443f, br); bi = fmaf(d9.y, 0.9646356105804443f, bi);
    ar = fmaf(s10.x, -0.956400990486145f, ar); ai = fmaf(s10.y, -0.956400990486145f, ai); br = fmaf(d10.x, 0.29205676913261414f, br); bi = fmaf(d10.y, 0.29205676913261414f, bi);
    ar = fmaf(s11.x, -0.3202698528766632f, ar); ai = fmaf(s11.y, -0.3202698528766632f, ai); br = fmaf(d11.x, -0.9473263621330261f, br); bi = fmaf(d11.y, -0.9473263621330261f, bi);
    ar = fmaf(s12.x, 0.9374196529388428f, ar); ai = fmaf(s12.y, 0.9374196529388428f, ai); br = fmaf(d12.x, -0.3482016324996948f, br); bi = fmaf(d12.y, -0.3482016324996948f, bi);
    ar = fmaf(s13.x, 0.3758275806903839f, ar); ai = fmaf(s13.y, 0.3758275806903839f, ai); br = fmaf(d13.x, 0.926689624786377f, br); bi = fmaf(d13.y, 0.926689624786377f, bi);
    ar = fmaf(s14.x, -0.9151456356048584f, ar); ai = fmaf(s14.y, -0.9151456356048584f, ai); br = fmaf(d14.x, 0.4031234383583069f, br); bi = fmaf(d14.y, 0.4031234383583069f, bi);
    ar = fmaf(s15.x, -0.43006521463394165f, ar); ai = fmaf(s15.y, -0.43006521463394165f, ai); br = fmaf(d15.x, -0.9027978181838989f, br); bi = fmaf(d15.y, -0.9027978181838989f, bi);
    ar = fmaf(s16.x, 0.8896570801734924f, ar); ai = fmaf(s16.y, 0.8896570801734924f, ai); br = fmaf(d16.x, -0.4566292464733124f, br); bi = fmaf(d16.y, -0.4566292464733124f, bi);
    ar = fmaf(s17.x, 0.4827921986579895f, ar); ai = fmaf(s17.y, 0.4827921986579895f, ai); br = fmaf(d17.x, 0.8757349252700806f, br); bi = fmaf(d17.y, 0.8757349252700806f, bi);
    ar = fmaf(s18.x, -0.8610436320304871f, ar); ai = fmaf(s18.y, -0.8610436320304871f, ai); br = fmaf(d18.x, 0.5085310935974121f, br); bi = fmaf(d18.y, 0.5085310935974121f, bi);
    ar = fmaf(s19.x, -0.5338233709335327f, ar); ai = fmaf(s19.y, -0.5338233709335327f, ai); br = fmaf(d19.x, -0.8455960154533386f, br); bi = fmaf(d19.y, -0.8455960154533386f, bi);
    ar = fmaf(s20.x, 0.829405665397644f, ar); ai = fmaf(s20.y, 0.829405665397644f, ai); br = fmaf(d20.x, -0.5586467385292053f, br); bi = fmaf(d20.y, -0.5586467385292053f, bi);
    ar = fmaf(s21.x, 0.5829795002937317f, ar); ai = fmaf(s21.y, 0.5829795002937317f, ai); br = fmaf(d21.x, 0.8124868869781494f, br); bi = fmaf(d21.y, 0.8124868869781494f, bi);
    ar = fmaf(s22.x, -0.794854462146759f, ar); ai = fmaf(s22.y, -0.794854462146759f, ai); br = fmaf(d22.x, 0.6068001389503479f, br); bi = fmaf(d22.y, 0.6068001389503479f, bi);
    ar = fmaf(s23.x, -0.6300878524780273f, ar); ai = fmaf(s23.y, -0.6300878524780273f, ai); br = fmaf(d23.x, -0.7765238881111145f, br); bi = fmaf(d23.y, -0.7765238881111145f, bi);
    ar = fmaf(s24.x, 0.7575112581253052f, ar); ai = fmaf(s24.y, 0.7575112581253052f, ai); br = fmaf(d24.x, -0.6528221368789673f, br); bi = fmaf(d24.y, -0.6528221368789673f, bi);
    ar = fmaf(s25.x, 0.674983024597168f, ar); ai = fmaf(s25.y, 0.674983024597168f, ai); br = fmaf(d25.x, 0.7378332614898682f, br); bi = fmaf(d25.y, 0.7378332614898682f, bi);
    ar = fmaf(s26.x, -0.7175072431564331f, ar); ai = fmaf(s26.y, -0.7175072431564331f, ai); br = fmaf(d26.x, 0.6965510249137878f, br); bi = fmaf(d26.y, 0.6965510249137878f, bi);
    if (!INV) {
      v[13] = make_float2(ar + bi, ai - br); v[40] = make_float2(ar - bi, ai + br);
    } else {
      v[13] = make_float2(ar - bi, ai + br); v[40] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.08879589289426804f, ar); ai = fmaf(s1.y, -0.08879589289426804f, ai); br = fmaf(d1.x, 0.9960498213768005f, br); bi = fmaf(d1.y, 0.9960498213768005f, bi);
    ar = fmaf(s2.x, -0.9842305779457092f, ar); ai = fmaf(s2.y, -0.9842305779457092f, ai); br = fmaf(d2.x, -0.1768902689218521f, br); bi = fmaf(d2.y, -0.1768902689218521f, bi);
    ar = fmaf(s3.x, 0.26358717679977417f, ar); ai = fmaf(s3.y, 0.26358717679977417f, ai); br = fmaf(d3.x, -0.9646356105804443f, br); bi = fmaf(d3.y, -0.9646356105804443f, bi);
    ar = fmaf(s4.x, 0.9374196529388428f, ar); ai = fmaf(s4.y, 0.9374196529388428f, ai); br = fmaf(d4.x, 0.3482016324996948f, br); bi = fmaf(d4.y, 0.3482016324996948f, bi);
    ar = fmaf(s5.x, -0.43006521463394165f, ar); ai = fmaf(s5.y, -0.43006521463394165f, ai); br = fmaf(d5.x, 0.9027978181838989f, br); bi = fmaf(d5.y, 0.9027978181838989f, bi);
    ar = fmaf(s6.x, -0.8610436320304871f, ar); ai = fmaf(s6.y, -0.8610436320304871f, ai); br = fmaf(d6.x, -0.5085310935974121f, br); bi = fmaf(d6.y, -0.5085310935974121f, bi);
    ar = fmaf(s7.x, 0.5829795002937317f, ar); ai = fmaf(s7.y, 0.5829795002937317f, ai); br = fmaf(d7.x, -0.8124868869781494f, br); bi = fmaf(d7.y, -0.8124868869781494f, bi);
    ar = fmaf(s8.x, 0.7575112581253052f, ar); ai = fmaf(s8.y, 0.7575112581253052f, ai); br = fmaf(d8.x, 0.6528221368789673f, br); bi = fmaf(d8.y, 0.6528221368789673f, bi);
    ar = fmaf(s9.x, -0.7175072431564331f, ar); ai = fmaf(s9.y, -0.7175072431564331f, ai); br = fmaf(d9.x, 0.6965510249137878f, br); bi = fmaf(d9.y, 0.6965510249137878f, bi);
    ar = fmaf(s10.x, -0.6300878524780273f, ar); ai = fmaf(s10.y, -0.6300878524780273f, ai); br = fmaf(d10.x, -0.7765238881111145f, br); bi = fmaf(d10.y, -0.7765238881111145f, bi);
    ar = fmaf(s11.x, 0.829405665397644f, ar); ai = fmaf(s11.y, 0.829405665397644f, ai); br = fmaf(d11.x, -0.5586467385292053f, br); bi = fmaf(d11.y, -0.5586467385292053f, bi);
    ar = fmaf(s12.x, 0.4827921986579895f, ar); ai = fmaf(s12.y, 0.4827921986579895f, ai); br = fmaf(d12.x, 0.8757349252700806f, br); bi = fmaf(d12.y, 0.8757349252700806f, bi);
    ar = fmaf(s13.x, -0.9151456356048584f, ar); ai = fmaf(s13.y, -0.9151456356048584f, ai); br = fmaf(d13.x, 0.4031234383583069f, br); bi = fmaf(d13.y, 0.4031234383583069f, bi);
    ar = fmaf(s14.x, -0.3202698528766632f, ar); ai = fmaf(s14.y, -0.3202698528766632f, ai); br = fmaf(d14.x, -0.9473263621330261f, br); bi = fmaf(d14.y, -0.9473263621330261f, bi);
    ar = fmaf(s15.x, 0.9720228910446167f, ar); ai = fmaf(s15.y, 0.9720228910446167f, ai); br = fmaf(d15.x, -0.2348860502243042f, br); bi = fmaf(d15.y, -0.2348860502243042f, bi);
    ar = fmaf(s16.x, 0.14764656126499176f, ar); ai = fmaf(s16.y, 0.14764656126499176f, ai); br = fmaf(d16.x, 0.989040195941925f, br); bi = fmaf(d16.y, 0.989040195941925f, bi);
    ar = fmaf(s17.x, -0.9982437491416931f, ar); ai = fmaf(s17.y, -0.9982437491416931f, ai); br = fmaf(d17.x, 0.05924062803387642f, br); bi = fmaf(d17.y, 0.05924062803387642f, bi);
    ar = fmaf(s18.x, 0.029633328318595886f, ar); ai = fmaf(s18.y, 0.029633328318595886f, ai); br = fmaf(d18.x, -0.9995608329772949f, br); bi = fmaf(d18.y, -0.9995608329772949f, bi);
    ar = fmaf(s19.x, 0.9929810762405396f, ar); ai = fmaf(s19.y, 0.9929810762405396f, ai); br = fmaf(d19.x, 0.11827316880226135f, br); bi = fmaf(d19.y, 0.11827316880226135f, bi);
    ar = fmaf(s20.x, -0.2059786170721054f, ar); ai = fmaf(s20.y, -0.2059786170721054f, ai); br = fmaf(d20.x, 0.9785565137863159f, br); bi = fmaf(d20.y, 0.9785565137863159f, bi);
    ar = fmaf(s21.x, -0.956400990486145f, ar); ai = fmaf(s21.y, -0.956400990486145f, ai); br = fmaf(d21.x, -0.29205676913261414f, br); bi = fmaf(d21.y, -0.29205676913261414f, bi);
    ar = fmaf(s22.x, 0.3758275806903839f, ar); ai = fmaf(s22.y, 0.3758275806903839f, ai); br = fmaf(d22.x, -0.926689624786377f, br); bi = fmaf(d22.y, -0.926689624786377f, bi);
    ar = fmaf(s23.x, 0.8896570801734924f, ar); ai = fmaf(s23.y, 0.8896570801734924f, ai); br = fmaf(d23.x, 0.4566292464733124f, br); bi = fmaf(d23.y, 0.4566292464733124f, bi);
    ar = fmaf(s24.x, -0.5338233709335327f, ar); ai = fmaf(s24.y, -0.5338233709335327f, ai); br = fmaf(d24.x, 0.8455960154533386f, br); bi = fmaf(d24.y, 0.8455960154533386f, bi);
    ar = fmaf(s25.x, -0.794854462146759f, ar); ai = fmaf(s25.y, -0.794854462146759f, ai); br = fmaf(d25.x, -0.6068001389503479f, br); bi = fmaf(d25.y, -0.6068001389503479f, bi);
    ar = fmaf(s26.x, 0.674983024597168f, ar); ai = fmaf(s26.y, 0.674983024597168f, ai); br = fmaf(d26.x, -0.7378332614898682f, br); bi = fmaf(d26.y, -0.7378332614898682f, bi);
    if (!INV) {
      v[14] = make_float2(ar + bi, ai - br); v[39] = make_float2(ar - bi, ai + br);
    } else {
      v[14] = make_float2(ar - bi, ai + br); v[39] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.2059786170721054f, ar); ai = fmaf(s1.y, -0.2059786170721054f, ai); br = fmaf(d1.x, 0.9785565137863159f, br); bi = fmaf(d1.y, 0.9785565137863159f, bi);
    ar = fmaf(s2.x, -0.9151456356048584f, ar); ai = fmaf(s2.y, -0.9151456356048584f, ai); br = fmaf(d2.x, -0.4031234383583069f, br); bi = fmaf(d2.y, -0.4031234383583069f, bi);
    ar = fmaf(s3.x, 0.5829795002937317f, ar); ai = fmaf(s3.y, 0.5829795002937317f, ai); br = fmaf(d3.x, -0.8124868869781494f, br); bi = fmaf(d3.y, -0.8124868869781494f, bi);
    ar = fmaf(s4.x, 0.674983024597168f, ar); ai = fmaf(s4.y, 0.674983024597168f, ai); br = fmaf(d4.x, 0.7378332614898682f, br); bi = fmaf(d4.y, 0.7378332614898682f, bi);
    ar = fmaf(s5.x, -0.8610436320304871f, ar); ai = fmaf(s5.y, -0.8610436320304871f, ai); br = fmaf(d5.x, 0.5085310935974121f, br); bi = fmaf(d5.y, 0.5085310935974121f, bi);
    ar = fmaf(s6.x, -0.3202698528766632f, ar); ai = fmaf(s6.y, -0.3202698528766632f, ai); br = fmaf(d6.x, -0.9473263621330261f, br); bi = fmaf(d6.y, -0.9473263621330261f, bi);
    ar = fmaf(s7.x, 0.9929810762405396f, ar); ai = fmaf(s7.y, 0.9929810762405396f, ai); br = fmaf(d7.x, -0.11827316880226135f, br); bi = fmaf(d7.y, -0.11827316880226135f, bi);
    ar = fmaf(s8.x, -0.08879589289426804f, ar); ai = fmaf(s8.y, -0.08879589289426804f, ai); br = fmaf(d8.x, 0.9960498213768005f, br); bi = fmaf(d8.y, 0.9960498213768005f, bi);
    ar = fmaf(s9.x, -0.956400990486145f, ar); ai = fmaf(s9.y, -0.956400990486145f, ai); br = fmaf(d9.x, -0.29205676913261414f, br); bi = fmaf(d9.y, -0.29205676913261414f, bi);
    ar = fmaf(s10.x, 0.4827921986579895f, ar); ai = fmaf(s10.y, 0.4827921986579895f, ai); br = fmaf(d10.x, -0.8757349252700806f, br); bi = fmaf(d10.y, -0.8757349252700806f, bi);
    ar = fmaf(s11.x, 0.7575112581253052f, ar); ai = fmaf(s11.y, 0.7575112581253052f, ai); br = fmaf(d11.x, 0.6528221368789673f, br); bi = fmaf(d11.y, 0.6528221368789673f, bi);
    ar = fmaf(s12.x, -0.794854462146759f, ar); ai = fmaf(s12.y, -0.794854462146759f, ai); br = fmaf(d12.x, 0.6068001389503479f, br); bi = fmaf(d12.y, 0.6068001389503479f, bi);
    ar = fmaf(s13.x, -0.43006521463394165f, ar); ai = fmaf(s13.y, -0.43006521463394165f, ai); br = fmaf(d13.x, -0.9027978181838989f, br); bi = fmaf(d13.y, -0.9027978181838989f, bi);
    ar = fmaf(s14.x, 0.9720228910446167f, ar); ai = fmaf(s14.y, 0.9720228910446167f, ai); br = fmaf(d14.x, -0.2348860502243042f, br); bi = fmaf(d14.y, -0.2348860502243042f, bi);
    ar = fmaf(s15.x, 0.029633328318595886f, ar); ai = fmaf(s15.y, 0.029633328318595886f, ai); br = fmaf(d15.x, 0.9995608329772949f, br); bi = fmaf(d15.y, 0.9995608329772949f, bi);
    ar = fmaf(s16.x, -0.9842305779457092f, ar); ai = fmaf(s16.y, -0.9842305779457092f, ai); br = fmaf(d16.x, -0.1768902689218521f, br); bi = fmaf(d16.y, -0.1768902689218521f, bi);
    ar = fmaf(s17.x, 0.3758275806903839f, ar); ai = fmaf(s17.y, 0.3758275806903839f, ai); br = fmaf(d17.x, -0.926689624786377f, br); bi = fmaf(d17.y, -0.926689624786377f, bi);
    ar = fmaf(s18.x, 0.829405665397644f, ar); ai = fmaf(s18.y, 0.829405665397644f, ai); br = fmaf(d18.x, 0.5586467385292053f, br); bi = fmaf(d18.y, 0.5586467385292053f, bi);
    ar = fmaf(s19.x, -0.7175072431564331f, ar); ai = fmaf(s19.y, -0.7175072431564331f, ai); br = fmaf(d19.x, 0.6965510249137878f, br); bi = fmaf(d19.y, 0.6965510249137878f, bi);
    ar = fmaf(s20.x, -0.5338233709335327f, ar); ai = fmaf(s20.y, -0.5338233709335327f, ai); br = fmaf(d20.x, -0.8455960154533386f, br); bi = fmaf(d20.y, -0.8455960154533386f, bi);
    ar = fmaf(s21.x, 0.9374196529388428f, ar); ai = fmaf(s21.y, 0.9374196529388428f, ai); br = fmaf(d21.x, -0.3482016324996948f, br); bi = fmaf(d21.y, -0.3482016324996948f, bi);
    ar = fmaf(s22.x, 0.14764656126499176f, ar); ai = fmaf(s22.y, 0.14764656126499176f, ai); br = fmaf(d22.x, 0.989040195941925f, br); bi = fmaf(d22.y, 0.989040195941925f, bi);
    ar = fmaf(s23.x, -0.9982437491416931f, ar); ai = fmaf(s23.y, -0.9982437491416931f, ai); br = fmaf(d23.x, -0.05924062803387642f, br); bi = fmaf(d23.y, -0.05924062803387642f, bi);
    ar = fmaf(s24.x, 0.26358717679977417f, ar); ai = fmaf(s24.y, 0.26358717679977417f, ai); br = fmaf(d24.x, -0.9646356105804443f, br); bi = fmaf(d24.y, -0.9646356105804443f, bi);
    ar = fmaf(s25.x, 0.8896570801734924f, ar); ai = fmaf(s25.y, 0.8896570801734924f, ai); br = fmaf(d25.x, 0.4566292464733124f, br); bi = fmaf(d25.y, 0.4566292464733124f, bi);
    ar = fmaf(s26.x, -0.6300878524780273f, ar); ai = fmaf(s26.y, -0.6300878524780273f, ai); br = fmaf(d26.x, 0.7765238881111145f, br); bi = fmaf(d26.y, 0.7765238881111145f, bi);
    if (!INV) {
      v[15] = make_float2(ar + bi, ai - br); v[38] = make_float2(ar - bi, ai + br);
    } else {
      v[15] = make_float2(ar - bi, ai + br); v[38] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.3202698528766632f, ar); ai = fmaf(s1.y, -0.3202698528766632f, ai); br = fmaf(d1.x, 0.9473263621330261f, br); bi = fmaf(d1.y, 0.9473263621330261f, bi);
    ar = fmaf(s2.x, -0.794854462146759f, ar); ai = fmaf(s2.y, -0.794854462146759f, ai); br = fmaf(d2.x, -0.6068001389503479f, br); bi = fmaf(d2.y, -0.6068001389503479f, bi);
    ar = fmaf(s3.x, 0.829405665397644f, ar); ai = fmaf(s3.y, 0.829405665397644f, ai); br = fmaf(d3.x, -0.5586467385292053f, br); bi = fmaf(d3.y, -0.5586467385292053f, bi);
    ar = fmaf(s4.x, 0.26358717679977417f, ar); ai = fmaf(s4.y, 0.26358717679977417f, ai); br = fmaf(d4.x, 0.9646356105804443f, br); bi = fmaf(d4.y, 0.9646356105804443f, bi);
    ar = fmaf(s5.x, -0.9982437491416931f, ar); ai = fmaf(s5.y, -0.9982437491416931f, ai); br = fmaf(d5.x, -0.05924062803387642f, br); bi = fmaf(d5.y, -0.05924062803387642f, bi);
    ar = fmaf(s6.x, 0.3758275806903839f, ar); ai = fmaf(s6.y, 0.3758275806903839f, ai); br = fmaf(d6.x, -0.926689624786377f, br); bi = fmaf(d6.y, -0.926689624786377f, bi);
    ar = fmaf(s7.x, 0.7575112581253052f, ar); ai = fmaf(s7.y, 0.7575112581253052f, ai); br = fmaf(d7.x, 0.6528221368789673f, br); bi = fmaf(d7.y, 0.6528221368789673f, bi);
    ar = fmaf(s8.x, -0.8610436320304871f, ar); ai = fmaf(s8.y, -0.8610436320304871f, ai); br = fmaf(d8.x, 0.5085310935974121f, br); bi = fmaf(d8.y, 0.5085310935974121f, bi);
    ar = fmaf(s9.x, -0.2059786170721054f, ar); ai = fmaf(s9.y, -0.2059786170721054f, ai); br = fmaf(d9.x, -0.9785565137863159f, br); bi = fmaf(d9.y, -0.9785565137863159f, bi);
    ar = fmaf(s10.x, 0.9929810762405396f, ar); ai = fmaf(s10.y, 0.9929810762405396f, ai); br = fmaf(d10.x, 0.11827316880226135f, br); bi = fmaf(d10.y, 0.11827316880226135f, bi);
    ar = fmaf(s11.x, -0.43006521463394165f, ar); ai = fmaf(s11.y, -0.43006521463394165f, ai); br = fmaf(d11.x, 0.9027978181838989f, br); bi = fmaf(d11.y, 0.9027978181838989f, bi);
    ar = fmaf(s12.x, -0.7175072431564331f, ar); ai = fmaf(s12.y, -0.7175072431564331f, ai); br = fmaf(d12.x, -0.6965510249137878f, br); bi = fmaf(d12.y, -0.6965510249137878f, bi);
    ar = fmaf(s13.x, 0.8896570801734924f, ar); ai = fmaf(s13.y, 0.8896570801734924f, ai); br = fmaf(d13.x, -0.4566292464733124f, br); bi = fmaf(d13.y, -0.4566292464733124f, bi);
    ar = fmaf(s14.x, 0.14764656126499176f, ar); ai = fmaf(s14.y, 0.14764656126499176f, ai); br = fmaf(d14.x, 0.989040195941925f, br); bi = fmaf(d14.y, 0.989040195941925f, bi);
    ar = fmaf(s15.x, -0.9842305779457092f, ar); ai = fmaf(s15.y, -0.9842305779457092f, ai); br = fmaf(d15.x, -0.1768902689218521f, br); bi = fmaf(d15.y, -0.1768902689218521f, bi);
    ar = fmaf(s16.x, 0.4827921986579895f, ar); ai = fmaf(s16.y, 0.4827921986579895f, ai); br = fmaf(d16.x, -0.8757349252700806f, br); bi = fmaf(d16.y, -0.8757349252700806f, bi);
    ar = fmaf(s17.x, 0.674983024597168f, ar); ai = fmaf(s17.y, 0.674983024597168f, ai); br = fmaf(d17.x, 0.7378332614898682f, br); bi = fmaf(d17.y, 0.7378332614898682f, bi);
    ar = fmaf(s18.x, -0.9151456356048584f, ar); ai = fmaf(s18.y, -0.9151456356048584f, ai); br = fmaf(d18.x, 0.4031234383583069f, br); bi = fmaf(d18.y, 0.4031234383583069f, bi);
    ar = fmaf(s19.x, -0.08879589289426804f, ar); ai = fmaf(s19.y, -0.08879589289426804f, ai); br = fmaf(d19.x, -0.9960498213768005f, br); bi = fmaf(d19.y, -0.9960498213768005f, bi);
    ar = fmaf(s20.x, 0.9720228910446167f, ar); ai = fmaf(s20.y, 0.9720228910446167f, ai); br = fmaf(d20.x, 0.2348860502243042f, br); bi = fmaf(d20.y, 0.2348860502243042f, bi);
    ar = fmaf(s21.x, -0.5338233709335327f, ar); ai = fmaf(s21.y, -0.5338233709335327f, ai); br = fmaf(d21.x, 0.8455960154533386f, br); bi = fmaf(d21.y, 0.8455960154533386f, bi);
    ar = fmaf(s22.x, -0.6300878524780273f, ar); ai = fmaf(s22.y, -0.6300878524780273f, ai); br = fmaf(d22.x, -0.7765238881111145f, br); bi = fmaf(d22.y, -0.7765238881111145f, bi);
    ar = fmaf(s23.x, 0.9374196529388428f, ar); ai = fmaf(s23.y, 0.9374196529388428f, ai); br = fmaf(d23.x, -0.3482016324996948f, br); bi = fmaf(d23.y, -0.3482016324996948f, bi);
    ar = fmaf(s24.x, 0.029633328318595886f, ar); ai = fmaf(s24.y, 0.029633328318595886f, ai); br = fmaf(d24.x, 0.9995608329772949f, br); bi = fmaf(d24.y, 0.9995608329772949f, bi);
    ar = fmaf(s25.x, -0.956400990486145f, ar); ai = fmaf(s25.y, -0.956400990486145f, ai); br = fmaf(d25.x, -0.29205676913261414f, br); bi = fmaf(d25.y, -0.29205676913261414f, bi);
    ar = fmaf(s26.x, 0.5829795002937317f, ar); ai = fmaf(s26.y, 0.5829795002937317f, ai); br = fmaf(d26.x, -0.8124868869781494f, br); bi = fmaf(d26.y, -0.8124868869781494f, bi);
    if (!INV) {
      v[16] = make_float2(ar + bi, ai - br); v[37] = make_float2(ar - bi, ai + br);
    } else {
      v[16] = make_float2(ar - bi, ai + br); v[37] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.43006521463394165f, ar); ai = fmaf(s1.y, -0.43006521463394165f, ai); br = fmaf(d1.x, 0.9027978181838989f, br); bi = fmaf(d1.y, 0.9027978181838989f, bi);
    ar = fmaf(s2.x, -0.6300878524780273f, ar); ai = fmaf(s2.y, -0.6300878524780273f, ai); br = fmaf(d2.x, -0.7765238881111145f, br); bi = fmaf(d2.y, -0.7765238881111145f, bi);
    ar = fmaf(s3.x, 0.9720228910446167f, ar); ai = fmaf(s3.y, 0.9720228910446167f, ai); br = fmaf(d3.x, -0.2348860502243042f, br); bi = fmaf(d3.y, -0.2348860502243042f, bi);
    ar = fmaf(s4.x, -0.2059786170721054f, ar); ai = fmaf(s4.y, -0.2059786170721054f, ai); br = fmaf(d4.x, 0.9785565137863159f, br); bi = fmaf(d4.y, 0.9785565137863159f, bi);
    ar = fmaf(s5.x, -0.794854462146759f, ar); ai = fmaf(s5.y, -0.794854462146759f, ai); br = fmaf(d5.x, -0.6068001389503479f, br); bi = fmaf(d5.y, -0.6068001389503479f, bi);
    ar = fmaf(s6.x, 0.8896570801734924f, ar); ai = fmaf(s6.y, 0.8896570801734924f, ai); br = fmaf(d6.x, -0.4566292464733124f, br); bi = fmaf(d6.y, -0.4566292464733124f, bi);
    ar = fmaf(s7.x, 0.029633328318595886f, ar); ai = fmaf(s7.y, 0.029633328318595886f, ai); br = fmaf(d7.x, 0.9995608329772949f, br); bi = fmaf(d7.y, 0.9995608329772949f, bi);
    ar = fmaf(s8.x, -0.9151456356048584f, ar); ai = fmaf(s8.y, -0.9151456356048584f, ai); br = fmaf(d8.x, -0.4031234383583069f, br); bi = fmaf(d8.y, -0.4031234383583069f, bi);
    ar = fmaf(s9.x, 0.7575112581253052f, ar); ai = fmaf(s9.y, 0.7575112581253052f, ai); br = fmaf(d9.x, -0.6528221368789673f, br); bi = fmaf(d9.y, -0.6528221368789673f, bi);
    ar = fmaf(s10.x, 0.26358717679977417f, ar); ai = fmaf(s10.y, 0.26358717679977417f, ai); br = fmaf(d10.x, 0.9646356105804443f, br); bi = fmaf(d10.y, 0.9646356105804443f, bi);
    ar = fmaf(s11.x, -0.9842305779457092f, ar); ai = fmaf(s11.y, -0.9842305779457092f, ai); br = fmaf(d11.x, -0.1768902689218521f, br); bi = fmaf(d11.y, -0.1768902689218521f, bi);
    ar = fmaf(s12.x, 0.5829795002937317f, ar); ai = fmaf(s12.y, 0.5829795002937317f, ai); br = fmaf(d12.x, -0.8124868869781494f, br); bi = fmaf(d12.y, -0.8124868869781494f, bi);
    ar = fmaf(s13.x, 0.4827921986579895f, ar); ai = fmaf(s13.y, 0.4827921986579895f, ai); br = fmaf(d13.x, 0.8757349252700806f, br); bi = fmaf(d13.y, 0.8757349252700806f, bi);
    ar = fmaf(s14.x, -0.9982437491416931f, ar); ai = fmaf(s14.y, -0.9982437491416931f, ai); br = fmaf(d14.x, 0.05924062803387642f, br); bi = fmaf(d14.y, 0.05924062803387642f, bi);
    ar = fmaf(s15.x, 0.3758275806903839f, ar); ai = fmaf(s15.y, 0.3758275806903839f, ai); br = fmaf(d15.x, -0.926689624786377f, br); bi = fmaf(d15.y, -0.926689624786377f, bi);
    ar = fmaf(s16.x, 0.674983024597168f, ar); ai = fmaf(s16.y, 0.674983024597168f, ai); br = fmaf(d16.x, 0.7378332614898682f, br); bi = fmaf(d16.y, 0.7378332614898682f, bi);
    ar = fmaf(s17.x, -0.956400990486145f, ar); ai = fmaf(s17.y, -0.956400990486145f, ai); br = fmaf(d17.x, 0.29205676913261414f, br); bi = fmaf(d17.y, 0.29205676913261414f, bi);
    ar = fmaf(s18.x, 0.14764656126499176f, ar); ai = fmaf(s18.y, 0.14764656126499176f, ai); br = fmaf(d18.x, -0.989040195941925f, br); bi = fmaf(d18.y, -0.989040195941925f, bi);
    ar = fmaf(s19.x, 0.829405665397644f, ar); ai = fmaf(s19.y, 0.829405665397644f, ai); br = fmaf(d19.x, 0.5586467385292053f, br); bi = fmaf(d19.y, 0.5586467385292053f, bi);
    ar = fmaf(s20.x, -0.8610436320304871f, ar); ai = fmaf(s20.y, -0.8610436320304871f, ai); br = fmaf(d20.x, 0.5085310935974121f, br); bi = fmaf(d20.y, 0.5085310935974121f, bi);
    ar = fmaf(s21.x, -0.08879589289426804f, ar); ai = fmaf(s21.y, -0.08879589289426804f, ai); br = fmaf(d21.x, -0.9960498213768005f, br); bi = fmaf(d21.y, -0.9960498213768005f, bi);
    ar = fmaf(s22.x, 0.9374196529388428f, ar); ai = fmaf(s22.y, 0.9374196529388428f, ai); br = fmaf(d22.x, 0.3482016324996948f, br); bi = fmaf(d22.y, 0.3482016324996948f, bi);
    ar = fmaf(s23.x, -0.7175072431564331f, ar); ai = fmaf(s23.y, -0.7175072431564331f, ai); br = fmaf(d23.x, 0.6965510249137878f, br); bi = fmaf(d23.y, 0.6965510249137878f, bi);
    ar = fmaf(s24.x, -0.3202698528766632f, ar); ai = fmaf(s24.y, -0.3202698528766632f, ai); br = fmaf(d24.x, -0.9473263621330261f, br); bi = fmaf(d24.y, -0.9473263621330261f, bi);
    ar = fmaf(s25.x, 0.9929810762405396f, ar); ai = fmaf(s25.y, 0.9929810762405396f, ai); br = fmaf(d25.x, 0.11827316880226135f, br); bi = fmaf(d25.y, 0.11827316880226135f, bi);
    ar = fmaf(s26.x, -0.5338233709335327f, ar); ai = fmaf(s26.y, -0.5338233709335327f, ai); br = fmaf(d26.x, 0.8455960154533386f, br); bi = fmaf(d26.y, 0.8455960154533386f, bi);
    if (!INV) {
      v[17] = make_float2(ar + bi, ai - br); v[36] = make_float2(ar - bi, ai + br);
    } else {
      v[17] = make_float2(ar - bi, ai + br); v[36] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.5338233709335327f, ar); ai = fmaf(s1.y, -0.5338233709335327f, ai); br = fmaf(d1.x, 0.8455960154533386f, br); bi = fmaf(d1.y, 0.8455960154533386f, bi);
    ar = fmaf(s2.x, -0.43006521463394165f, ar); ai = fmaf(s2.y, -0.43006521463394165f, ai); br = fmaf(d2.x, -0.9027978181838989f, br); bi = fmaf(d2.y, -0.9027978181838989f, bi);
    ar = fmaf(s3.x, 0.9929810762405396f, ar); ai = fmaf(s3.y, 0.9929810762405396f, ai); br = fmaf(d3.x, 0.11827316880226135f, br); bi = fmaf(d3.y, 0.11827316880226135f, bi);
    ar = fmaf(s4.x, -0.6300878524780273f, ar); ai = fmaf(s4.y, -0.6300878524780273f, ai); br = fmaf(d4.x, 0.7765238881111145f, br); bi = fmaf(d4.y, 0.7765238881111145f, bi);
    ar = fmaf(s5.x, -0.3202698528766632f, ar); ai = fmaf(s5.y, -0.3202698528766632f, ai); br = fmaf(d5.x, -0.9473263621330261f, br); bi = fmaf(d5.y, -0.9473263621330261f, bi);
    ar = fmaf(s6.x, 0.9720228910446167f, ar); ai = fmaf(s6.y, 0.9720228910446167f, ai); br = fmaf(d6.x, 0.2348860502243042f, br); bi = fmaf(d6.y, 0.2348860502243042f, bi);
    ar = fmaf(s7.x, -0.7175072431564331f, ar); ai = fmaf(s7.y, -0.7175072431564331f, ai); br = fmaf(d7.x, 0.6965510249137878f, br); bi = fmaf(d7.y, 0.6965510249137878f, bi);
    ar = fmaf(s8.x, -0.2059786170721054f, ar); ai = fmaf(s8.y, -0.2059786170721054f, ai); br = fmaf(d8.x, -0.9785565137863159f, br); bi = fmaf(d8.y, -0.9785565137863159f, bi);
    ar = fmaf(s9.x, 0.9374196529388428f, ar); ai = fmaf(s9.y, 0.9374196529388428f, ai); br = fmaf(d9.x, 0.3482016324996948f, br); bi = fmaf(d9.y, 0.3482016324996948f, bi);
    ar = fmaf(s10.x, -0.794854462146759f, ar); ai = fmaf(s10.y, -0.794854462146759f, ai); br = fmaf(d10.x, 0.6068001389503479f, br); bi = fmaf(d10.y, 0.6068001389503479f, bi);
    ar = fmaf(s11.x, -0.08879589289426804f, ar); ai = fmaf(s11.y, -0.08879589289426804f, ai); br = fmaf(d11.x, -0.9960498213768005f, br); bi = fmaf(d11.y, -0.9960498213768005f, bi);
    ar = fmaf(s12.x, 0.8896570801734924f, ar); ai = fmaf(s12.y, 0.8896570801734924f, ai); br = fmaf(d12.x, 0.4566292464733124f, br); bi = fmaf(d12.y, 0.4566292464733124f, bi);
    ar = fmaf(s13.x, -0.8610436320304871f, ar); ai = fmaf(s13.y, -0.8610436320304871f, ai); br = fmaf(d13.x, 0.5085310935974121f, br); bi = fmaf(d13.y, 0.5085310935974121f, bi);
    ar = fmaf(s14.x, 0.029633328318595886f, ar); ai = fmaf(s14.y, 0.029633328318595886f, ai); br = fmaf(d14.x, -0.9995608329772949f, br); bi = fmaf(d14.y, -0.9995608329772949f, bi);
    ar = fmaf(s15.x, 0.829405665397644f, ar); ai = fmaf(s15.y, 0.829405665397644f, ai); br = fmaf(d15.x, 0.5586467385292053f, br); bi = fmaf(d15.y, 0.5586467385292053f, bi);
    ar = fmaf(s16.x, -0.9151456356048584f, ar); ai = fmaf(s16.y, -0.9151456356048584f, ai); br = fmaf(d16.x, 0.4031234383583069f, br); bi = fmaf(d16.y, 0.4031234383583069f, bi);
    ar = fmaf(s17.x, 0.14764656126499176f, ar); ai = fmaf(s17.y, 0.14764656126499176f, ai); br = fmaf(d17.x, -0.989040195941925f, br); bi = fmaf(d17.y, -0.989040195941925f, bi);
    ar = fmaf(s18.x, 0.7575112581253052f, ar); ai = fmaf(s18.y, 0.7575112581253052f, ai); br = fmaf(d18.x, 0.6528221368789673f, br); bi = fmaf(d18.y, 0.6528221368789673f, bi);
    ar = fmaf(s19.x, -0.956400990486145f, ar); ai = fmaf(s19.y, -0.956400990486145f, ai); br = fmaf(d19.x, 0.29205676913261414f, br); bi = fmaf(d19.y, 0.29205676913261414f, bi);
    ar = fmaf(s20.x, 0.26358717679977417f, ar); ai = fmaf(s20.y, 0.26358717679977417f, ai); br = fmaf(d20.x, -0.9646356105804443f, br); bi = fmaf(d20.y, -0.9646356105804443f, bi);
    ar = fmaf(s21.x, 0.674983024597168f, ar); ai = fmaf(s21.y, 0.674983024597168f, ai); br = fmaf(d21.x, 0.7378332614898682f, br); bi = fmaf(d21.y, 0.7378332614898682f, bi);
    ar = fmaf(s22.x, -0.9842305779457092f, ar); ai = fmaf(s22.y, -0.9842305779457092f, ai); br = fmaf(d22.x, 0.1768902689218521f, br); bi = fmaf(d22.y, 0.1768902689218521f, bi);
    ar = fmaf(s23.x, 0.3758275806903839f, ar); ai = fmaf(s23.y, 0.3758275806903839f, ai); br = fmaf(d23.x, -0.926689624786377f, br); bi = fmaf(d23.y, -0.926689624786377f, bi);
    ar = fmaf(s24.x, 0.5829795002937317f, ar); ai = fmaf(s24.y, 0.5829795002937317f, ai); br = fmaf(d24.x, 0.8124868869781494f, br); bi = fmaf(d24.y, 0.8124868869781494f, bi);
    ar = fmaf(s25.x, -0.9982437491416931f, ar); ai = fmaf(s25.y, -0.9982437491416931f, ai); br = fmaf(d25.x, 0.05924062803387642f, br); bi = fmaf(d25.y, 0.05924062803387642f, bi);
    ar = fmaf(s26.x, 0.4827921986579895f, ar); ai = fmaf(s26.y, 0.4827921986579895f, ai); br = fmaf(d26.x, -0.8757349252700806f, br); bi = fmaf(d26.y, -0.8757349252700806f, bi);
    if (!INV) {
      v[18] = make_float2(ar + bi, ai - br); v[35] = make_float2(ar - bi, ai + br);
    } else {
      v[18] = make_float2(ar - bi, ai + br); v[35] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.6300878524780273f, ar); ai = fmaf(s1.y, -0.6300878524780273f, ai); br = fmaf(d1.x, 0.7765238881111145f, br); bi = fmaf(d1.y, 0.7765238881111145f, bi);
    ar = fmaf(s2.x, -0.2059786170721054f, ar); ai = fmaf(s2.y, -0.2059786170721054f, ai); br = fmaf(d2.x, -0.9785565137863159f, br); bi = fmaf(d2.y, -0.9785565137863159f, bi);
    ar = fmaf(s3.x, 0.8896570801734924f, ar); ai = fmaf(s3.y, 0.8896570801734924f, ai); br = fmaf(d3.x, 0.4566292464733124f, br); bi = fmaf(d3.y, 0.4566292464733124f, bi);
    ar = fmaf(s4.x, -0.9151456356048584f, ar); ai = fmaf(s4.y, -0.9151456356048584f, ai); br = fmaf(d4.x, 0.4031234383583069f, br); bi = fmaf(d4.y, 0.4031234383583069f, bi);
    ar = fmaf(s5.x, 0.26358717679977417f, ar); ai = fmaf(s5.y, 0.26358717679977417f, ai); br = fmaf(d5.x, -0.9646356105804443f, br); bi = fmaf(d5.y, -0.9646356105804443f, bi);
    ar = fmaf(s6.x, 0.5829795002937317f, ar); ai = fmaf(s6.y, 0.5829795002937317f, ai); br = fmaf(d6.x, 0.8124868869781494f, br); bi = fmaf(d6.y, 0.8124868869781494f, bi);
    ar = fmaf(s7.x, -0.9982437491416931f, ar); ai = fmaf(s7.y, -0.9982437491416931f, ai); br = fmaf(d7.x, -0.05924062803387642f, br); bi = fmaf(d7.y, -0.05924062803387642f, bi);
    ar = fmaf(s8.x, 0.674983024597168f, ar); ai = fmaf(s8.y, 0.674983024597168f, ai); br = fmaf(d8.x, -0.7378332614898682f, br); bi = fmaf(d8.y, -0.7378332614898682f, bi);
    ar = fmaf(s9.x, 0.14764656126499176f, ar); ai = fmaf(s9.y, 0.14764656126499176f, ai); br = fmaf(d9.x, 0.989040195941925f, br); bi = fmaf(d9.y, 0.989040195941925f, bi);
    ar = fmaf(s10.x, -0.8610436320304871f, ar); ai = fmaf(s10.y, -0.8610436320304871f, ai); br = fmaf(d10.x, -0.5085310935974121f, br); bi = fmaf(d10.y, -0.5085310935974121f, bi);
    ar = fmaf(s11.x, 0.9374196529388428f, ar); ai = fmaf(s11.y, 0.9374196529388428f, ai); br = fmaf(d11.x, -0.3482016324996948f, br); bi = fmaf(d11.y, -0.3482016324996948f, bi);
    ar = fmaf(s12.x, -0.3202698528766632f, ar); ai = fmaf(s12.y, -0.3202698528766632f, ai); br = fmaf(d12.x, 0.9473263621330261f, br); bi = fmaf(d12.y, 0.9473263621330261f, bi);
    ar = fmaf(s13.x, -0.5338233709335327f, ar); ai = fmaf(s13.y, -0.5338233709335327f, ai); br = fmaf(d13.x, -0.8455960154533386f, br); bi = fmaf(d13.y, -0.8455960154533386f, bi);
    ar = fmaf(s14.x, 0.9929810762405396f, ar); ai = fmaf(s14.y, 0.9929810762405396f, ai); br = fmaf(d14.x, 0.11827316880226135f, br); bi = fmaf(d14.y, 0.11827316880226135f, bi);
    ar = fmaf(s15.x, -0.7175072431564331f, ar); ai = fmaf(s15.y, -0.7175072431564331f, ai); br = fmaf(d15.x, 0.6965510249137878f, br); bi = fmaf(d15.y, 0.6965510249137878f, bi);
    ar = fmaf(s16.x, -0.08879589289426804f, ar); ai = fmaf(s16.y, -0.08879589289426804f, ai); br = fmaf(d16.x, -0.9960498213768005f, br); bi = fmaf(d16.y, -0.9960498213768005f, bi);
    ar = fmaf(s17.x, 0.829405665397644f, ar); ai = fmaf(s17.y, 0.829405665397644f, ai); br = fmaf(d17.x, 0.5586467385292053f, br); bi = fmaf(d17.y, 0.5586467385292053f, bi);
    ar = fmaf(s18.x, -0.956400990486145f, ar); ai = fmaf(s18.y, -0.956400990486145f, ai); br = fmaf(d18.x, 0.29205676913261414f, br); bi = fmaf(d18.y, 0.29205676913261414f, bi);
    ar = fmaf(s19.x, 0.3758275806903839f, ar); ai = fmaf(s19.y, 0.3758275806903839f, ai); br = fmaf(d19.x, -0.926689624786377f, br); bi = fmaf(d19.y, -0.926689624786377f, bi);
    ar = fmaf(s20.x, 0.4827921986579895f, ar); ai = fmaf(s20.y, 0.4827921986579895f, ai); br = fmaf(d20.x, 0.8757349252700806f, br); bi = fmaf(d20.y, 0.8757349252700806f, bi);
    ar = fmaf(s21.x, -0.9842305779457092f, ar); ai = fmaf(s21.y, -0.9842305779457092f, ai); br = fmaf(d21.x, -0.1768902689218521f, br); bi = fmaf(d21.y, -0.1768902689218521f, bi);
    ar = fmaf(s22.x, 0.7575112581253052f, ar); ai = fmaf(s22.y, 0.7575112581253052f, ai); br = fmaf(d22.x, -0.6528221368789673f, br); bi = fmaf(d22.y, -0.6528221368789673f, bi);
    ar = fmaf(s23.x, 0.029633328318595886f, ar); ai = fmaf(s23.y, 0.029633328318595886f, ai); br = fmaf(d23.x, 0.9995608329772949f, br); bi = fmaf(d23.y, 0.9995608329772949f, bi);
    ar = fmaf(s24.x, -0.794854462146759f, ar); ai = fmaf(s24.y, -0.794854462146759f, ai); br = fmaf(d24.x, -0.6068001389503479f, br); bi = fmaf(d24.y, -0.6068001389503479f, bi);
    ar = fmaf(s25.x, 0.9720228910446167f, ar); ai = fmaf(s25.y, 0.9720228910446167f, ai); br = fmaf(d25.x, -0.2348860502243042f, br); bi = fmaf(d25.y, -0.2348860502243042f, bi);
    ar = fmaf(s26.x, -0.43006521463394165f, ar); ai = fmaf(s26.y, -0.43006521463394165f, ai); br = fmaf(d26.x, 0.9027978181838989f, br); bi = fmaf(d26.y, 0.9027978181838989f, bi);
    if (!INV) {
      v[19] = make_float2(ar + bi, ai - br); v[34] = make_float2(ar - bi, ai + br);
    } else {
      v[19] = make_float2(ar - bi, ai + br); v[34] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.7175072431564331f, ar); ai = fmaf(s1.y, -0.7175072431564331f, ai); br = fmaf(d1.x, 0.6965510249137878f, br); bi = fmaf(d1.y, 0.6965510249137878f, bi);
    ar = fmaf(s2.x, 0.029633328318595886f, ar); ai = fmaf(s2.y, 0.029633328318595886f, ai); br = fmaf(d2.x, -0.9995608329772949f, br); bi = fmaf(d2.y, -0.9995608329772949f, bi);
    ar = fmaf(s3.x, 0.674983024597168f, ar); ai = fmaf(s3.y, 0.674983024597168f, ai); br = fmaf(d3.x, 0.7378332614898682f, br); bi = fmaf(d3.y, 0.7378332614898682f, bi);
    ar = fmaf(s4.x, -0.9982437491416931f, ar); ai = fmaf(s4.y, -0.9982437491416931f, ai); br = fmaf(d4.x, -0.05924062803387642f, br); bi = fmaf(d4.y, -0.05924062803387642f, bi);
    ar = fmaf(s5.x, 0.7575112581253052f, ar); ai = fmaf(s5.y, 0.7575112581253052f, ai); br = fmaf(d5.x, -0.6528221368789673f, br); bi = fmaf(d5.y, -0.6528221368789673f, bi);
    ar = fmaf(s6.x, -0.08879589289426804f, ar); ai = fmaf(s6.y, -0.08879589289426804f, ai); br = fmaf(d6.x, 0.9960498213768005f, br); bi = fmaf(d6.y, 0.9960498213768005f, bi);
    ar = fmaf(s7.x, -0.6300878524780273f, ar); ai = fmaf(s7.y, -0.6300878524780273f, ai); br = fmaf(d7.x, -0.7765238881111145f, br); bi = fmaf(d7.y, -0.7765238881111145f, bi);
    ar = fmaf(s8.x, 0.9929810762405396f, ar); ai = fmaf(s8.y, 0.9929810762405396f, ai); br = fmaf(d8.x, 0.11827316880226135f, br); bi = fmaf(d8.y, 0.11827316880226135f, bi);
    ar = fmaf(s9.x, -0.794854462146759f, ar); ai = fmaf(s9.y, -0.794854462146759f, ai); br = fmaf(d9.x, 0.6068001389503479f, br); bi = fmaf(d9.y, 0.6068001389503479f, bi);
    ar = fmaf(s10.x, 0.14764656126499176f, ar); ai = fmaf(s10.y, 0.14764656126499176f, ai); br = fmaf(d10.x, -0.989040195941925f, br); bi = fmaf(d10.y, -0.989040195941925f, bi);
    ar = fmaf(s11.x, 0.5829795002937317f, ar); ai = fmaf(s11.y, 0.5829795002937317f, ai); br = fmaf(d11.x, 0.8124868869781494f, br); bi = fmaf(d11.y, 0.8124868869781494f, bi);
    ar = fmaf(s12.x, -0.9842305779457092f, ar); ai = fmaf(s12.y, -0.9842305779457092f, ai); br = fmaf(d12.x, -0.1768902689218521f, br); bi = fmaf(d12.y, -0.1768902689218521f, bi);
    ar = fmaf(s13.x, 0.829405665397644f, ar); ai = fmaf(s13.y, 0.829405665397644f, ai); br = fmaf(d13.x, -0.5586467385292053f, br); bi = fmaf(d13.y, -0.5586467385292053f, bi);
    ar = fmaf(s14.x, -0.2059786170721054f, ar); ai = fmaf(s14.y, -0.2059786170721054f, ai); br = fmaf(d14.x, 0.9785565137863159f, br); bi = fmaf(d14.y, 0.9785565137863159f, bi);
    ar = fmaf(s15.x, -0.5338233709335327f, ar); ai = fmaf(s15.y, -0.5338233709335327f, ai); br = fmaf(d15.x, -0.8455960154533386f, br); bi = fmaf(d15.y, -0.8455960154533386f, bi);
    ar = fmaf(s16.x, 0.9720228910446167f, ar); ai = fmaf(s16.y, 0.9720228910446167f, ai); br = fmaf(d16.x, 0.2348860502243042f, br); bi = fmaf(d16.y, 0.2348860502243042f, bi);
    ar = fmaf(s17.x, -0.8610436320304871f, ar); ai = fmaf(s17.y, -0.8610436320304871f, ai); br = fmaf(d17.x, 0.5085310935974121f, br); bi = fmaf(d17.y, 0.5085310935974121f, bi);
    ar = fmaf(s18.x, 0.26358717679977417f, ar); ai = fmaf(s18.y, 0.26358717679977417f, ai); br = fmaf(d18.x, -0.9646356105804443f, br); bi = fmaf(d18.y, -0.9646356105804443f, bi);
    ar = fmaf(s19.x, 0.4827921986579895f, ar); ai = fmaf(s19.y, 0.4827921986579895f, ai); br = fmaf(d19.x, 0.8757349252700806f, br); bi = fmaf(d19.y, 0.8757349252700806f, bi);
    ar = fmaf(s20.x, -0.956400990486145f, ar); ai = fmaf(s20.y, -0.956400990486145f, ai); br = fmaf(d20.x, -0.29205676913261414f, br); bi = fmaf(d20.y, -0.29205676913261414f, bi);
    ar = fmaf(s21.x, 0.8896570801734924f, ar); ai = fmaf(s21.y, 0.8896570801734924f, ai); br = fmaf(d21.x, -0.4566292464733124f, br); bi = fmaf(d21.y, -0.4566292464733124f, bi);
    ar = fmaf(s22.x, -0.3202698528766632f, ar); ai = fmaf(s22.y, -0.3202698528766632f, ai); br = fmaf(d22.x, 0.9473263621330261f, br); bi = fmaf(d22.y, 0.9473263621330261f, bi);
    ar = fmaf(s23.x, -0.43006521463394165f, ar); ai = fmaf(s23.y, -0.43006521463394165f, ai); br = fmaf(d23.x, -0.9027978181838989f, br); bi = fmaf(d23.y, -0.9027978181838989f, bi);
    ar = fmaf(s24.x, 0.9374196529388428f, ar); ai = fmaf(s24.y, 0.9374196529388428f, ai); br = fmaf(d24.x, 0.3482016324996948f, br); bi = fmaf(d24.y, 0.3482016324996948f, bi);
    ar = fmaf(s25.x, -0.9151456356048584f, ar); ai = fmaf(s25.y, -0.9151456356048584f, ai); br = fmaf(d25.x, 0.4031234383583069f, br); bi = fmaf(d25.y, 0.4031234383583069f, bi);
    ar = fmaf(s26.x, 0.3758275806903839f, ar); ai = fmaf(s26.y, 0.3758275806903839f, ai); br = fmaf(d26.x, -0.926689624786377f, br); bi = fmaf(d26.y, -0.926689624786377f, bi);
    if (!INV) {
      v[20] = make_float2(ar + bi, ai - br); v[33] = make_float2(ar - bi, ai + br);
    } else {
      v[20] = make_float2(ar - bi, ai + br); v[33] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.794854462146759f, ar); ai = fmaf(s1.y, -0.794854462146759f, ai); br = fmaf(d1.x, 0.6068001389503479f, br); bi = fmaf(d1.y, 0.6068001389503479f, bi);
    ar = fmaf(s2.x, 0.26358717679977417f, ar); ai = fmaf(s2.y, 0.26358717679977417f, ai); br = fmaf(d2.x, -0.9646356105804443f, br); bi = fmaf(d2.y, -0.9646356105804443f, bi);
    ar = fmaf(s3.x, 0.3758275806903839f, ar); ai = fmaf(s3.y, 0.3758275806903839f, ai); br = fmaf(d3.x, 0.926689624786377f, br); bi = fmaf(d3.y, 0.926689624786377f, bi);
    ar = fmaf(s4.x, -0.8610436320304871f, ar); ai = fmaf(s4.y, -0.8610436320304871f, ai); br = fmaf(d4.x, -0.5085310935974121f, br); bi = fmaf(d4.y, -0.5085310935974121f, bi);
    ar = fmaf(s5.x, 0.9929810762405396f, ar); ai = fmaf(s5.y, 0.9929810762405396f, ai); br = fmaf(d5.x, -0.11827316880226135f, br); bi = fmaf(d5.y, -0.11827316880226135f, bi);
    ar = fmaf(s6.x, -0.7175072431564331f, ar); ai = fmaf(s6.y, -0.7175072431564331f, ai); br = fmaf(d6.x, 0.6965510249137878f, br); bi = fmaf(d6.y, 0.6965510249137878f, bi);
    ar = fmaf(s7.x, 0.14764656126499176f, ar); ai = fmaf(s7.y, 0.14764656126499176f, ai); br = fmaf(d7.x, -0.989040195941925f, br); bi = fmaf(d7.y, -0.989040195941925f, bi);
    ar = fmaf(s8.x, 0.4827921986579895f, ar); ai = fmaf(s8.y, 0.4827921986579895f, ai); br = fmaf(d8.x, 0.8757349252700806f, br); bi = fmaf(d8.y, 0.8757349252700806f, bi);
    ar = fmaf(s9.x, -0.9151456356048584f, ar); ai = fmaf(s9.y, -0.9151456356048584f, ai); br = fmaf(d9.x, -0.4031234383583069f, br); bi = fmaf(d9.y, -0.4031234383583069f, bi);
    ar = fmaf(s10.x, 0.9720228910446167f, ar); ai = fmaf(s10.y, 0.9720228910446167f, ai); br = fmaf(d10.x, -0.2348860502243042f, br); bi = fmaf(d10.y, -0.2348860502243042f, bi);
    ar = fmaf(s11.x, -0.6300878524780273f, ar); ai = fmaf(s11.y, -0.6300878524780273f, ai); br = fmaf(d11.x, 0.7765238881111145f, br); bi = fmaf(d11.y, 0.7765238881111145f, bi);
    ar = fmaf(s12.x, 0.029633328318595886f, ar); ai = fmaf(s12.y, 0.029633328318595886f, ai); br = fmaf(d12.x, -0.9995608329772949f, br); bi = fmaf(d12.y, -0.9995608329772949f, bi);
    ar = fmaf(s13.x, 0.5829795002937317f, ar); ai = fmaf(s13.y, 0.5829795002937317f, ai); br = fmaf(d13.x, 0.8124868869781494f, br); bi = fmaf(d13.y, 0.8124868869781494f, bi);
    ar = fmaf(s14.x, -0.956400990486145f, ar); ai = fmaf(s14.y, -0.956400990486145f, ai); br = fmaf(d14.x, -0.29205676913261414f, br); bi = fmaf(d14.y, -0.29205676913261414f, bi);
    ar = fmaf(s15.x, 0.9374196529388428f, ar); ai = fmaf(s15.y, 0.9374196529388428f, ai); br = fmaf(d15.x, -0.3482016324996948f, br); bi = fmaf(d15.y, -0.3482016324996948f, bi);
    ar = fmaf(s16.x, -0.5338233709335327f, ar); ai = fmaf(s16.y, -0.5338233709335327f, ai); br = fmaf(d16.x, 0.8455960154533386f, br); bi = fmaf(d16.y, 0.8455960154533386f, bi);
    ar = fmaf(s17.x, -0.08879589289426804f, ar); ai = fmaf(s17.y, -0.08879589289426804f, ai); br = fmaf(d17.x, -0.9960498213768005f, br); bi = fmaf(d17.y, -0.9960498213768005f, bi);
    ar = fmaf(s18.x, 0.674983024597168f, ar); ai = fmaf(s18.y, 0.674983024597168f, ai); br = fmaf(d18.x, 0.7378332614898682f, br); bi = fmaf(d18.y, 0.7378332614898682f, bi);
    ar = fmaf(s19.x, -0.9842305779457092f, ar); ai = fmaf(s19.y, -0.9842305779457092f, ai); br = fmaf(d19.x, -0.1768902689218521f, br); bi = fmaf(d19.y, -0.1768902689218521f, bi);
    ar = fmaf(s20.x, 0.8896570801734924f, ar); ai = fmaf(s20.y, 0.8896570801734924f, ai); br = fmaf(d20.x, -0.4566292464733124f, br); bi = fmaf(d20.y, -0.4566292464733124f, bi);
    ar = fmaf(s21.x, -0.43006521463394165f, ar); ai = fmaf(s21.y, -0.43006521463394165f, ai); br = fmaf(d21.x, 0.9027978181838989f, br); bi = fmaf(d21.y, 0.9027978181838989f, bi);
    ar = fmaf(s22.x, -0.2059786170721054f, ar); ai = fmaf(s22.y, -0.2059786170721054f, ai); br = fmaf(d22.x, -0.9785565137863159f, br); bi = fmaf(d22.y, -0.9785565137863159f, bi);
    ar = fmaf(s23.x, 0.7575112581253052f, ar); ai = fmaf(s23.y, 0.7575112581253052f, ai); br = fmaf(d23.x, 0.6528221368789673f, br); bi = fmaf(d23.y, 0.6528221368789673f, bi);
    ar = fmaf(s24.x, -0.9982437491416931f, ar); ai = fmaf(s24.y, -0.9982437491416931f, ai); br = fmaf(d24.x, -0.05924062803387642f, br); bi = fmaf(d24.y, -0.05924062803387642f, bi);
    ar = fmaf(s25.x, 0.829405665397644f, ar); ai = fmaf(s25.y, 0.829405665397644f, ai); br = fmaf(d25.x, -0.5586467385292053f, br); bi = fmaf(d25.y, -0.5586467385292053f, bi);
    ar = fmaf(s26.x, -0.3202698528766632f, ar); ai = fmaf(s26.y, -0.3202698528766632f, ai); br = fmaf(d26.x, 0.9473263621330261f, br); bi = fmaf(d26.y, 0.9473263621330261f, bi);
    if (!INV) {
      v[21] = make_float2(ar + bi, ai - br); v[32] = make_float2(ar - bi, ai + br);
    } else {
      v[21] = make_float2(ar - bi, ai + br); v[32] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.8610436320304871f, ar); ai = fmaf(s1.y, -0.8610436320304871f, ai); br = fmaf(d1.x, 0.5085310935974121f, br); bi = fmaf(d1.y, 0.5085310935974121f, bi);
    ar = fmaf(s2.x, 0.4827921986579895f, ar); ai = fmaf(s2.y, 0.4827921986579895f, ai); br = fmaf(d2.x, -0.8757349252700806f, br); bi = fmaf(d2.y, -0.8757349252700806f, bi);
    ar = fmaf(s3.x, 0.029633328318595886f, ar); ai = fmaf(s3.y, 0.029633328318595886f, ai); br = fmaf(d3.x, 0.9995608329772949f, br); bi = fmaf(d3.y, 0.9995608329772949f, bi);
    ar = fmaf(s4.x, -0.5338233709335327f, ar); ai = fmaf(s4.y, -0.5338233709335327f, ai); br = fmaf(d4.x, -0.8455960154533386f, br); bi = fmaf(d4.y, -0.8455960154533386f, bi);
    ar = fmaf(s5.x, 0.8896570801734924f, ar); ai = fmaf(s5.y, 0.8896570801734924f, ai); br = fmaf(d5.x, 0.4566292464733124f, br); bi = fmaf(d5.y, 0.4566292464733124f, bi);
    ar = fmaf(s6.x, -0.9982437491416931f, ar); ai = fmaf(s6.y, -0.9982437491416931f, ai); br = fmaf(d6.x, 0.05924062803387642f, br); bi = fmaf(d6.y, 0.05924062803387642f, bi);
    ar = fmaf(s7.x, 0.829405665397644f, ar); ai = fmaf(s7.y, 0.829405665397644f, ai); br = fmaf(d7.x, -0.5586467385292053f, br); bi = fmaf(d7.y, -0.5586467385292053f, bi);
    ar = fmaf(s8.x, -0.43006521463394165f, ar); ai = fmaf(s8.y, -0.43006521463394165f, ai); br = fmaf(d8.x, 0.9027978181838989f, br); bi = fmaf(d8.y, 0.9027978181838989f, bi);
    ar = fmaf(s9.x, -0.08879589289426804f, ar); ai = fmaf(s9.y, -0.08879589289426804f, ai); br = fmaf(d9.x, -0.9960498213768005f, br); bi = fmaf(d9.y, -0.9960498213768005f, bi);
    ar = fmaf(s10.x, 0.5829795002937317f, ar); ai = fmaf(s10.y, 0.5829795002937317f, ai); br = fmaf(d10.x, 0.8124868869781494f, br); bi = fmaf(d10.y, 0.8124868869781494f, bi);
    ar = fmaf(s11.x, -0.9151456356048584f, ar); ai = fmaf(s11.y, -0.9151456356048584f, ai); br = fmaf(d11.x, -0.4031234383583069f, br); bi = fmaf(d11.y, -0.4031234383583069f, bi);
    ar = fmaf(s12.x, 0.9929810762405396f, ar); ai = fmaf(s12.y, 0.9929810762405396f, ai); br = fmaf(d12.x, -0.11827316880226135f, br); bi = fmaf(d12.y, -0.11827316880226135f, bi);
    ar = fmaf(s13.x, -0.794854462146759f, ar); ai = fmaf(s13.y, -0.794854462146759f, ai); br = fmaf(d13.x, 0.6068001389503479f, br); bi = fmaf(d13.y, 0.6068001389503479f, bi);
    ar = fmaf(s14.x, 0.3758275806903839f, ar); ai = fmaf(s14.y, 0.3758275806903839f, ai); br = fmaf(d14.x, -0.926689624786377f, br); bi = fmaf(d14.y, -0.926689624786377f, bi);
    ar = fmaf(s15.x, 0.14764656126499176f, ar); ai = fmaf(s15.y, 0.14764656126499176f, ai); br = fmaf(d15.x, 0.989040195941925f, br); bi = fmaf(d15.y, 0.989040195941925f, bi);
    ar = fmaf(s16.x, -0.6300878524780273f, ar); ai = fmaf(s16.y, -0.6300878524780273f, ai); br = fmaf(d16.x, -0.7765238881111145f, br); bi = fmaf(d16.y, -0.7765238881111145f, bi);
    ar = fmaf(s17.x, 0.9374196529388428f, ar); ai = fmaf(s17.y, 0.9374196529388428f, ai); br = fmaf(d17.x, 0.3482016324996948f, br); bi = fmaf(d17.y, 0.3482016324996948f, bi);
    ar = fmaf(s18.x, -0.9842305779457092f, ar); ai = fmaf(s18.y, -0.9842305779457092f, ai); br = fmaf(d18.x, 0.1768902689218521f, br); bi = fmaf(d18.y, 0.1768902689218521f, bi);
    ar = fmaf(s19.x, 0.7575112581253052f, ar); ai = fmaf(s19.y, 0.7575112581253052f, ai); br = fmaf(d19.x, -0.6528221368789673f, br); bi = fmaf(d19.y, -0.6528221368789673f, bi);
    ar = fmaf(s20.x, -0.3202698528766632f, ar); ai = fmaf(s20.y, -0.3202698528766632f, ai); br = fmaf(d20.x, 0.9473263621330261f, br); bi = fmaf(d20.y, 0.9473263621330261f, bi);
    ar = fmaf(s21.x, -0.2059786170721054f, ar); ai = fmaf(s21.y, -0.2059786170721054f, ai); br = fmaf(d21.x, -0.9785565137863159f, br); bi = fmaf(d21.y, -0.9785565137863159f, bi);
    ar = fmaf(s22.x, 0.674983024597168f, ar); ai = fmaf(s22.y, 0.674983024597168f, ai); br = fmaf(d22.x, 0.7378332614898682f, br); bi = fmaf(d22.y, 0.7378332614898682f, bi);
    ar = fmaf(s23.x, -0.956400990486145f, ar); ai = fmaf(s23.y, -0.956400990486145f, ai); br = fmaf(d23.x, -0.29205676913261414f, br); bi = fmaf(d23.y, -0.29205676913261414f, bi);
    ar = fmaf(s24.x, 0.9720228910446167f, ar); ai = fmaf(s24.y, 0.9720228910446167f, ai); br = fmaf(d24.x, -0.2348860502243042f, br); bi = fmaf(d24.y, -0.2348860502243042f, bi);
    ar = fmaf(s25.x, -0.7175072431564331f, ar); ai = fmaf(s25.y, -0.7175072431564331f, ai); br = fmaf(d25.x, 0.6965510249137878f, br); bi = fmaf(d25.y, 0.6965510249137878f, bi);
    ar = fmaf(s26.x, 0.26358717679977417f, ar); ai = fmaf(s26.y, 0.26358717679977417f, ai); br = fmaf(d26.x, -0.9646356105804443f, br); bi = fmaf(d26.y, -0.9646356105804443f, bi);
    if (!INV) {
      v[22] = make_float2(ar + bi, ai - br); v[31] = make_float2(ar - bi, ai + br);
    } else {
      v[22] = make_float2(ar - bi, ai + br); v[31] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.9151456356048584f, ar); ai = fmaf(s1.y, -0.9151456356048584f, ai); br = fmaf(d1.x, 0.4031234383583069f, br); bi = fmaf(d1.y, 0.4031234383583069f, bi);
    ar = fmaf(s2.x, 0.674983024597168f, ar); ai = fmaf(s2.y, 0.674983024597168f, ai); br = fmaf(d2.x, -0.7378332614898682f, br); bi = fmaf(d2.y, -0.7378332614898682f, bi);
    ar = fmaf(s3.x, -0.3202698528766632f, ar); ai = fmaf(s3.y, -0.3202698528766632f, ai); br = fmaf(d3.x, 0.9473263621330261f, br); bi = fmaf(d3.y, 0.9473263621330261f, bi);
    ar = fmaf(s4.x, -0.08879589289426804f, ar); ai = fmaf(s4.y, -0.08879589289426804f, ai); br = fmaf(d4.x, -0.9960498213768005f, br); bi = fmaf(d4.y, -0.9960498213768005f, bi);
    ar = fmaf(s5.x, 0.4827921986579895f, ar); ai = fmaf(s5.y, 0.4827921986579895f, ai); br = fmaf(d5.x, 0.8757349252700806f, br); bi = fmaf(d5.y, 0.8757349252700806f, bi);
    ar = fmaf(s6.x, -0.794854462146759f, ar); ai = fmaf(s6.y, -0.794854462146759f, ai); br = fmaf(d6.x, -0.6068001389503479f, br); bi = fmaf(d6.y, -0.6068001389503479f, bi);
    ar = fmaf(s7.x, 0.9720228910446167f, ar); ai = fmaf(s7.y, 0.9720228910446167f, ai); br = fmaf(d7.x, 0.2348860502243042f, br); bi = fmaf(d7.y, 0.2348860502243042f, bi);
    ar = fmaf(s8.x, -0.9842305779457092f, ar); ai = fmaf(s8.y, -0.9842305779457092f, ai); br = fmaf(d8.x, 0.1768902689218521f, br); bi = fmaf(d8.y, 0.1768902689218521f, bi);
    ar = fmaf(s9.x, 0.829405665397644f, ar); ai = fmaf(s9.y, 0.829405665397644f, ai); br = fmaf(d9.x, -0.5586467385292053f, br); bi = fmaf(d9.y, -0.5586467385292053f, bi);
    ar = fmaf(s10.x, -0.5338233709335327f, ar); ai = fmaf(s10.y, -0.5338233709335327f, ai); br = fmaf(d10.x, 0.8455960154533386f, br); bi = fmaf(d10.y, 0.8455960154533386f, bi);
    ar = fmaf(s11.x, 0.14764656126499176f, ar); ai = fmaf(s11.y, 0.14764656126499176f, ai); br = fmaf(d11.x, -0.989040195941925f, br); bi = fmaf(d11.y, -0.989040195941925f, bi);
    ar = fmaf(s12.x, 0.26358717679977417f, ar); ai = fmaf(s12.y, 0.26358717679977417f, ai); br = fmaf(d12.x, 0.9646356105804443f, br); bi = fmaf(d12.y, 0.9646356105804443f, bi);
    ar = fmaf(s13.x, -0.6300878524780273f, ar); ai = fmaf(s13.y, -0.6300878524780273f, ai); br = fmaf(d13.x, -0.7765238881111145f, br); bi = fmaf(d13.y, -0.7765238881111145f, bi);
    ar = fmaf(s14.x, 0.8896570801734924f, ar); ai = fmaf(s14.y, 0.8896570801734924f, ai); br = fmaf(d14.x, 0.4566292464733124f, br); bi = fmaf(d14.y, 0.4566292464733124f, bi);
    ar = fmaf(s15.x, -0.9982437491416931f, ar); ai = fmaf(s15.y, -0.9982437491416931f, ai); br = fmaf(d15.x, -0.05924062803387642f, br); bi = fmaf(d15.y, -0.05924062803387642f, bi);
    ar = fmaf(s16.x, 0.9374196529388428f, ar); ai = fmaf(s16.y, 0.9374196529388428f, ai); br = fmaf(d16.x, -0.3482016324996948f, br); bi = fmaf(d16.y, -0.3482016324996948f, bi);
    ar = fmaf(s17.x, -0.7175072431564331f, ar); ai = fmaf(s17.y, -0.7175072431564331f, ai); br = fmaf(d17.x, 0.6965510249137878f, br); bi = fmaf(d17.y, 0.6965510249137878f, bi);
    ar = fmaf(s18.x, 0.3758275806903839f, ar); ai = fmaf(s18.y, 0.3758275806903839f, ai); br = fmaf(d18.x, -0.926689624786377f, br); bi = fmaf(d18.y, -0.926689624786377f, bi);
    ar = fmaf(s19.x, 0.029633328318595886f, ar); ai = fmaf(s19.y, 0.029633328318595886f, ai); br = fmaf(d19.x, 0.9995608329772949f, br); bi = fmaf(d19.y, 0.9995608329772949f, bi);
    ar = fmaf(s20.x, -0.43006521463394165f, ar); ai = fmaf(s20.y, -0.43006521463394165f, ai); br = fmaf(d20.x, -0.9027978181838989f, br); bi = fmaf(d20.y, -0.9027978181838989f, bi);
    ar = fmaf(s21.x, 0.7575112581253052f, ar); ai = fmaf(s21.y, 0.7575112581253052f, ai); br = fmaf(d21.x, 0.6528221368789673f, br); bi = fmaf(d21.y, 0.6528221368789673f, bi);
    ar = fmaf(s22.x, -0.956400990486145f, ar); ai = fmaf(s22.y, -0.956400990486145f, ai); br = fmaf(d22.x, -0.29205676913261414f, br); bi = fmaf(d22.y, -0.29205676913261414f, bi);
    ar = fmaf(s23.x, 0.9929810762405396f, ar); ai = fmaf(s23.y, 0.9929810762405396f, ai); br = fmaf(d23.x, -0.11827316880226135f, br); bi = fmaf(d23.y, -0.11827316880226135f, bi);
    ar = fmaf(s24.x, -0.8610436320304871f, ar); ai = fmaf(s24.y, -0.8610436320304871f, ai); br = fmaf(d24.x, 0.5085310935974121f, br); bi = fmaf(d24.y, 0.5085310935974121f, bi);
    ar = fmaf(s25.x, 0.5829795002937317f, ar); ai = fmaf(s25.y, 0.5829795002937317f, ai); br = fmaf(d25.x, -0.8124868869781494f, br); bi = fmaf(d25.y, -0.8124868869781494f, bi);
    ar = fmaf(s26.x, -0.2059786170721054f, ar); ai = fmaf(s26.y, -0.2059786170721054f, ai); br = fmaf(d26.x, 0.9785565137863159f, br); bi = fmaf(d26.y, 0.9785565137863159f, bi);
    if (!INV) {
      v[23] = make_float2(ar + bi, ai - br); v[30] = make_float2(ar - bi, ai + br);
    } else {
      v[23] = make_float2(ar - bi, ai + br); v[30] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.956400990486145f, ar); ai = fmaf(s1.y, -0.956400990486145f, ai); br = fmaf(d1.x, 0.29205676913261414f, br); bi = fmaf(d1.y, 0.29205676913261414f, bi);
    ar = fmaf(s2.x, 0.829405665397644f, ar); ai = fmaf(s2.y, 0.829405665397644f, ai); br = fmaf(d2.x, -0.5586467385292053f, br); bi = fmaf(d2.y, -0.5586467385292053f, bi);
    ar = fmaf(s3.x, -0.6300878524780273f, ar); ai = fmaf(s3.y, -0.6300878524780273f, ai); br = fmaf(d3.x, 0.7765238881111145f, br); bi = fmaf(d3.y, 0.7765238881111145f, bi);
    ar = fmaf(s4.x, 0.3758275806903839f, ar); ai = fmaf(s4.y, 0.3758275806903839f, ai); br = fmaf(d4.x, -0.926689624786377f, br); bi = fmaf(d4.y, -0.926689624786377f, bi);
    ar = fmaf(s5.x, -0.08879589289426804f, ar); ai = fmaf(s5.y, -0.08879589289426804f, ai); br = fmaf(d5.x, 0.9960498213768005f, br); bi = fmaf(d5.y, 0.9960498213768005f, bi);
    ar = fmaf(s6.x, -0.2059786170721054f, ar); ai = fmaf(s6.y, -0.2059786170721054f, ai); br = fmaf(d6.x, -0.9785565137863159f, br); bi = fmaf(d6.y, -0.9785565137863159f, bi);
    ar = fmaf(s7.x, 0.4827921986579895f, ar); ai = fmaf(s7.y, 0.4827921986579895f, ai); br = fmaf(d7.x, 0.8757349252700806f, br); bi = fmaf(d7.y, 0.8757349252700806f, bi);
    ar = fmaf(s8.x, -0.7175072431564331f, ar); ai = fmaf(s8.y, -0.7175072431564331f, ai); br = fmaf(d8.x, -0.6965510249137878f, br); bi = fmaf(d8.y, -0.6965510249137878f, bi);
    ar = fmaf(s9.x, 0.8896570801734924f, ar); ai = fmaf(s9.y, 0.8896570801734924f, ai); br = fmaf(d9.x, 0.4566292464733124f, br); bi = fmaf(d9.y, 0.4566292464733124f, bi);
    ar = fmaf(s10.x, -0.9842305779457092f, ar); ai = fmaf(s10.y, -0.9842305779457092f, ai); br = fmaf(d10.x, -0.1768902689218521f, br); bi = fmaf(d10.y, -0.1768902689218521f, bi);
    ar = fmaf(s11.x, 0.9929810762405396f, ar); ai = fmaf(s11.y, 0.9929810762405396f, ai); br = fmaf(d11.x, -0.11827316880226135f, br); bi = fmaf(d11.y, -0.11827316880226135f, bi);
    ar = fmaf(s12.x, -0.9151456356048584f, ar); ai = fmaf(s12.y, -0.9151456356048584f, ai); br = fmaf(d12.x, 0.4031234383583069f, br); bi = fmaf(d12.y, 0.4031234383583069f, bi);
    ar = fmaf(s13.x, 0.7575112581253052f, ar); ai = fmaf(s13.y, 0.7575112581253052f, ai); br = fmaf(d13.x, -0.6528221368789673f, br); bi = fmaf(d13.y, -0.6528221368789673f, bi);
    ar = fmaf(s14.x, -0.5338233709335327f, ar); ai = fmaf(s14.y, -0.5338233709335327f, ai); br = fmaf(d14.x, 0.8455960154533386f, br); bi = fmaf(d14.y, 0.8455960154533386f, bi);
    ar = fmaf(s15.x, 0.26358717679977417f, ar); ai = fmaf(s15.y, 0.26358717679977417f, ai); br = fmaf(d15.x, -0.9646356105804443f, br); bi = fmaf(d15.y, -0.9646356105804443f, bi);
    ar = fmaf(s16.x, 0.029633328318595886f, ar); ai = fmaf(s16.y, 0.029633328318595886f, ai); br = fmaf(d16.x, 0.9995608329772949f, br); bi = fmaf(d16.y, 0.9995608329772949f, bi);
    ar = fmaf(s17.x, -0.3202698528766632f, ar); ai = fmaf(s17.y, -0.3202698528766632f, ai); br = fmaf(d17.x, -0.9473263621330261f, br); bi = fmaf(d17.y, -0.9473263621330261f, bi);
    ar = fmaf(s18.x, 0.5829795002937317f, ar); ai = fmaf(s18.y, 0.5829795002937317f, ai); br = fmaf(d18.x, 0.8124868869781494f, br); bi = fmaf(d18.y, 0.8124868869781494f, bi);
    ar = fmaf(s19.x, -0.794854462146759f, ar); ai = fmaf(s19.y, -0.794854462146759f, ai); br = fmaf(d19.x, -0.6068001389503479f, br); bi = fmaf(d19.y, -0.6068001389503479f, bi);
    ar = fmaf(s20.x, 0.9374196529388428f, ar); ai = fmaf(s20.y, 0.9374196529388428f, ai); br = fmaf(d20.x, 0.3482016324996948f, br); bi = fmaf(d20.y, 0.3482016324996948f, bi);
    ar = fmaf(s21.x, -0.9982437491416931f, ar); ai = fmaf(s21.y, -0.9982437491416931f, ai); br = fmaf(d21.x, -0.05924062803387642f, br); bi = fmaf(d21.y, -0.05924062803387642f, bi);
    ar = fmaf(s22.x, 0.9720228910446167f, ar); ai = fmaf(s22.y, 0.9720228910446167f, ai); br = fmaf(d22.x, -0.2348860502243042f, br); bi = fmaf(d22.y, -0.2348860502243042f, bi);
    ar = fmaf(s23.x, -0.8610436320304871f, ar); ai = fmaf(s23.y, -0.8610436320304871f, ai); br = fmaf(d23.x, 0.5085310935974121f, br); bi = fmaf(d23.y, 0.5085310935974121f, bi);
    ar = fmaf(s24.x, 0.674983024597168f, ar); ai = fmaf(s24.y, 0.674983024597168f, ai); br = fmaf(d24.x, -0.7378332614898682f, br); bi = fmaf(d24.y, -0.7378332614898682f, bi);
    ar = fmaf(s25.x, -0.43006521463394165f, ar); ai = fmaf(s25.y, -0.43006521463394165f, ai); br = fmaf(d25.x, 0.9027978181838989f, br); bi = fmaf(d25.y, 0.9027978181838989f, bi);
    ar = fmaf(s26.x, 0.14764656126499176f, ar); ai = fmaf(s26.y, 0.14764656126499176f, ai); br = fmaf(d26.x, -0.989040195941925f, br); bi = fmaf(d26.y, -0.989040195941925f, bi);
    if (!INV) {
      v[24] = make_float2(ar + bi, ai - br); v[29] = make_float2(ar - bi, ai + br);
    } else {
      v[24] = make_float2(ar - bi, ai + br); v[29] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.9842305779457092f, ar); ai = fmaf(s1.y, -0.9842305779457092f, ai); br = fmaf(d1.x, 0.1768902689218521f, br); bi = fmaf(d1.y, 0.1768902689218521f, bi);
    ar = fmaf(s2.x, 0.9374196529388428f, ar); ai = fmaf(s2.y, 0.9374196529388428f, ai); br = fmaf(d2.x, -0.3482016324996948f, br); bi = fmaf(d2.y, -0.3482016324996948f, bi);
    ar = fmaf(s3.x, -0.8610436320304871f, ar); ai = fmaf(s3.y, -0.8610436320304871f, ai); br = fmaf(d3.x, 0.5085310935974121f, br); bi = fmaf(d3.y, 0.5085310935974121f, bi);
    ar = fmaf(s4.x, 0.7575112581253052f, ar); ai = fmaf(s4.y, 0.7575112581253052f, ai); br = fmaf(d4.x, -0.6528221368789673f, br); bi = fmaf(d4.y, -0.6528221368789673f, bi);
    ar = fmaf(s5.x, -0.6300878524780273f, ar); ai = fmaf(s5.y, -0.6300878524780273f, ai); br = fmaf(d5.x, 0.7765238881111145f, br); bi = fmaf(d5.y, 0.7765238881111145f, bi);
    ar = fmaf(s6.x, 0.4827921986579895f, ar); ai = fmaf(s6.y, 0.4827921986579895f, ai); br = fmaf(d6.x, -0.8757349252700806f, br); bi = fmaf(d6.y, -0.8757349252700806f, bi);
    ar = fmaf(s7.x, -0.3202698528766632f, ar); ai = fmaf(s7.y, -0.3202698528766632f, ai); br = fmaf(d7.x, 0.9473263621330261f, br); bi = fmaf(d7.y, 0.9473263621330261f, bi);
    ar = fmaf(s8.x, 0.14764656126499176f, ar); ai = fmaf(s8.y, 0.14764656126499176f, ai); br = fmaf(d8.x, -0.989040195941925f, br); bi = fmaf(d8.y, -0.989040195941925f, bi);
    ar = fmaf(s9.x, 0.029633328318595886f, ar); ai = fmaf(s9.y, 0.029633328318595886f, ai); br = fmaf(d9.x, 0.9995608329772949f, br); bi = fmaf(d9.y, 0.9995608329772949f, bi);
    ar = fmaf(s10.x, -0.2059786170721054f, ar); ai = fmaf(s10.y, -0.2059786170721054f, ai); br = fmaf(d10.x, -0.9785565137863159f, br); bi = fmaf(d10.y, -0.9785565137863159f, bi);
    ar = fmaf(s11.x, 0.3758275806903839f, ar); ai = fmaf(s11.y, 0.3758275806903839f, ai); br = fmaf(d11.x, 0.926689624786377f, br); bi = fmaf(d11.y, 0.926689624786377f, bi);
    ar = fmaf(s12.x, -0.5338233709335327f, ar); ai = fmaf(s12.y, -0.5338233709335327f, ai); br = fmaf(d12.x, -0.8455960154533386f, br); bi = fmaf(d12.y, -0.8455960154533386f, bi);
    ar = fmaf(s13.x, 0.674983024597168f, ar); ai = fmaf(s13.y, 0.674983024597168f, ai); br = fmaf(d13.x, 0.7378332614898682f, br); bi = fmaf(d13.y, 0.7378332614898682f, bi);
    ar = fmaf(s14.x, -0.794854462146759f, ar); ai = fmaf(s14.y, -0.794854462146759f, ai); br = fmaf(d14.x, -0.6068001389503479f, br); bi = fmaf(d14.y, -0.6068001389503479f, bi);
    ar = fmaf(s15.x, 0.8896570801734924f, ar); ai = fmaf(s15.y, 0.8896570801734924f, ai); br = fmaf(d15.x, 0.4566292464733124f, br); bi = fmaf(d15.y, 0.4566292464733124f, bi);
    ar = fmaf(s16.x, -0.956400990486145f, ar); ai = fmaf(s16.y, -0.956400990486145f, ai); br = fmaf(d16.x, -0.29205676913261414f, br); bi = fmaf(d16.y, -0.29205676913261414f, bi);
    ar = fmaf(s17.x, 0.9929810762405396f, ar); ai = fmaf(s17.y, 0.9929810762405396f, ai); br = fmaf(d17.x, 0.11827316880226135f, br); bi = fmaf(d17.y, 0.11827316880226135f, bi);
    ar = fmaf(s18.x, -0.9982437491416931f, ar); ai = fmaf(s18.y, -0.9982437491416931f, ai); br = fmaf(d18.x, 0.05924062803387642f, br); bi = fmaf(d18.y, 0.05924062803387642f, bi);
    ar = fmaf(s19.x, 0.9720228910446167f, ar); ai = fmaf(s19.y, 0.9720228910446167f, ai); br = fmaf(d19.x, -0.2348860502243042f, br); bi = fmaf(d19.y, -0.2348860502243042f, bi);
    ar = fmaf(s20.x, -0.9151456356048584f, ar); ai = fmaf(s20.y, -0.9151456356048584f, ai); br = fmaf(d20.x, 0.4031234383583069f, br); bi = fmaf(d20.y, 0.4031234383583069f, bi);
    ar = fmaf(s21.x, 0.829405665397644f, ar); ai = fmaf(s21.y, 0.829405665397644f, ai); br = fmaf(d21.x, -0.5586467385292053f, br); bi = fmaf(d21.y, -0.5586467385292053f, bi);
    ar = fmaf(s22.x, -0.7175072431564331f, ar); ai = fmaf(s22.y, -0.7175072431564331f, ai); br = fmaf(d22.x, 0.6965510249137878f, br); bi = fmaf(d22.y, 0.6965510249137878f, bi);
    ar = fmaf(s23.x, 0.5829795002937317f, ar); ai = fmaf(s23.y, 0.5829795002937317f, ai); br = fmaf(d23.x, -0.8124868869781494f, br); bi = fmaf(d23.y, -0.8124868869781494f, bi);
    ar = fmaf(s24.x, -0.43006521463394165f, ar); ai = fmaf(s24.y, -0.43006521463394165f, ai); br = fmaf(d24.x, 0.9027978181838989f, br); bi = fmaf(d24.y, 0.9027978181838989f, bi);
    ar = fmaf(s25.x, 0.26358717679977417f, ar); ai = fmaf(s25.y, 0.26358717679977417f, ai); br = fmaf(d25.x, -0.9646356105804443f, br); bi = fmaf(d25.y, -0.9646356105804443f, bi);
    ar = fmaf(s26.x, -0.08879589289426804f, ar); ai = fmaf(s26.y, -0.08879589289426804f, ai); br = fmaf(d26.x, 0.9960498213768005f, br); bi = fmaf(d26.y, 0.9960498213768005f, bi);
    if (!INV) {
      v[25] = make_float2(ar + bi, ai - br); v[28] = make_float2(ar - bi, ai + br);
    } else {
      v[25] = make_float2(ar - bi, ai + br); v[28] = make_float2(ar + bi, ai - br);
    }
  }
  {
    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
    ar = fmaf(s1.x, -0.9982437491416931f, ar); ai = fmaf(s1.y, -0.9982437491416931f, ai); br = fmaf(d1.x, 0.05924062803387642f, br); bi = fmaf(d1.y, 0.05924062803387642f, bi);
    ar = fmaf(s2.x, 0.9929810762405396f, ar); ai = fmaf(s2.y, 0.9929810762405396f, ai); br = fmaf(d2.x, -0.11827316880226135f, br); bi = fmaf(d2.y, -0.11827316880226135f, bi);
    ar = fmaf(s3.x, -0.9842305779457092f, ar); ai = fmaf(s3.y, -0.9842305779457092f, ai); br = fmaf(d3.x, 0.1768902689218521f, br); bi = fmaf(d3.y, 0.1768902689218521f, bi);
    ar = fmaf(s4.x, 0.9720228910446167f, ar); ai = fmaf(s4.y, 0.9720228910446167f, ai); br = fmaf(d4.x, -0.2348860502243042f, br); bi = fmaf(d4.y, -0.2348860502243042f, bi);
    ar = fmaf(s5.x, -0.956400990486145f, ar); ai = fmaf(s5.y, -0.956400990486145f, ai); br = fmaf(d5.x, 0.29205676913261414f, br); bi = fmaf(d5.y, 0.29205676913261414f, bi);
    ar = fmaf(s6.x, 0.9374196529388428f, ar); ai = fmaf(s6.y, 0.9374196529388428f, ai); br = fmaf(d6.x, -0.3482016324996948f, br); bi = fmaf(d6.y, -0.3482016324996948f, bi);
    ar = fmaf(s7.x, -0.9151456356048584f, ar); ai = fmaf(s7.y, -0.9151456356048584f, ai); br = fmaf(d7.x, 0.4031234383583069f, br); bi = fmaf(d7.y, 0.4031234383583069f, bi);
    ar = fmaf(s8.x, 0.8896570801734924f, ar); ai = fmaf(s8.y, 0.8896570801734924f, ai); br = fmaf(d8.x, -0.4566292464733124f, br); bi = fmaf(d8.y, -0.4566292464733124f, bi);
    ar = fmaf(s9.x, -0.8610436320304871f, ar); ai = fmaf(s9.y, -0.8610436320304871f, ai); br = fmaf(d9.x, 0.5085310935974121f, br); bi = fmaf(d9.y, 0.5085310935974121f, bi);
    ar = fmaf(s10.x, 0.829405665397644f, ar); ai = fmaf(s10.y, 0.829405665397644f, ai); br = fmaf(d10.x, -0.5586467385292053f, br); bi = fmaf(d10.y, -0.5586467385292053f, bi);
    ar = fmaf(s11.x, -0.794854462146759f, ar); ai = fmaf(s11.y, -0.794854462146759f, ai); br = fmaf(d11.x, 0.6068001389503479f, br); bi = fmaf(d11.y, 0.6068001389503479f, bi);
    ar = fmaf(s12.x, 0.7575112581253052f, ar); ai = fmaf(s12.y, 0.7575112581253052f, ai); br = fmaf(d12.x, -0.6528221368789673f, br); bi = fmaf(d12.y, -0.6528221368789673f, bi);
    ar = fmaf(s13.x, -0.7175072431564331f, ar); ai = fmaf(s13.y, -0.7175072431564331f, ai); br = fmaf(d13.x, 0.6965510249137878f, br); bi = fmaf(d13.y, 0.6965510249137878f, bi);
    ar = fmaf(s14.x, 0.674983024597168f, ar); ai = fmaf(s14.y, 0.674983024597168f, ai); br = fmaf(d14.x, -0.7378332614898682f, br); bi = fmaf(d14.y, -0.7378332614898682f, bi);
    ar = fmaf(s15.x, -0.6300878524780273f, ar); ai = fmaf(s15.y, -0.6300878524780273f, ai); br = fmaf(d15.x, 0.7765238881111145f, br); bi = fmaf(d15.y, 0.7765238881111145f, bi);
    ar = fmaf(s16.x, 0.5829795002937317f, ar); ai = fmaf(s16.y, 0.5829795002937317f, ai); br = fmaf(d16.x, -0.8124868869781494f, br); bi = fmaf(d16.y, -0.8124868869781494f, bi);
    ar = fmaf(s17.x, -0.5338233709335327f, ar); ai = fmaf(s17.y, -0.5338233709335327f, ai); br = fmaf(d17.x, 0.8455960154533386f, br); bi = fmaf(d17.y, 0.8455960154533386f, bi);
    ar = fmaf(s18.x, 0.4827921986579895f, ar); ai = fmaf(s18.y, 0.4827921986579895f, ai); br = fmaf(d18.x, -0.8757349252700806f, br); bi = fmaf(d18.y, -0.8757349252700806f, bi);
    ar = fmaf(s19.x, -0.43006521463394165f, ar); ai = fmaf(s19.y, -0.43006521463394165f, ai); br = fmaf(d19.x, 0.9027978181838989f, br); bi = fmaf(d19.y, 0.9027978181838989f, bi);
    ar = fmaf(s20.x, 0.3758275806903839f, ar); ai = fmaf(s20.y, 0.3758275806903839f, ai); br = fmaf(d20.x, -0.926689624786377f, br); bi = fmaf(d20.y, -0.926689624786377f, bi);
    ar = fmaf(s21.x, -0.3202698528766632f, ar); ai = fmaf(s21.y, -0.3202698528766632f, ai); br = fmaf(d21.x, 0.9473263621330261f, br); bi = fmaf(d21.y, 0.9473263621330261f, bi);
    ar = fmaf(s22.x, 0.26358717679977417f, ar); ai = fmaf(s22.y, 0.26358717679977417f, ai); br = fmaf(d22.x, -0.9646356105804443f, br); bi = fmaf(d22.y, -0.9646356105804443f, bi);
    ar = fmaf(s23.x, -0.2059786170721054f, ar); ai = fmaf(s23.y, -0.2059786170721054f, ai); br = fmaf(d23.x, 0.9785565137863159f, br); bi = fmaf(d23.y, 0.9785565137863159f, bi);
    ar = fmaf(s24.x, 0.14764656126499176f, ar); ai = fmaf(s24.y, 0.14764656126499176f, ai); br = fmaf(d24.x, -0.989040195941925f, br); bi = fmaf(d24.y, -0.989040195941925f, bi);
    ar = fmaf(s25.x, -0.08879589289426804f, ar); ai = fmaf(s25.y, -0.08879589289426804f, ai); br = fmaf(d25.x, 0.9960498213768005f, br); bi = fmaf(d25.y, 0.9960498213768005f, bi);
    ar = fmaf(s26.x, 0.029633328318595886f, ar); ai = fmaf(s26.y, 0.029633328318595886f, ai); br = fmaf(d26.x, -0.9995608329772949f, br); bi = fmaf(d26.y, -0.9995608329772949f, bi);
    if (!INV) {
      v[26] = make_float2(ar + bi, ai - br); v[27] = make_float2(ar - bi, ai + br);
    } else {
      v[26] = make_float2(ar - bi, ai + br); v[27] = make_float2(ar + bi, ai - br);
    }
  }
}
constexpr int kSplit53 = 3;
template <bool INV, typename St>
__device__ __forceinline__ void dft_r53_part(const float2* v, int part, St&& st) {
  const float2 x0 = v[0];
  const float2 s1 = padd(v[1], v[52]);
  const float2 d1 = psub(v[1], v[52]);
  const float2 s2 = padd(v[2], v[51]);
  const float2 d2 = psub(v[2], v[51]);
  const float2 s3 = padd(v[3], v[50]);
  const float2 d3 = psub(v[3], v[50]);
  const float2 s4 = padd(v[4], v[49]);
  const float2 d4 = psub(v[4], v[49]);
  const float2 s5 = padd(v[5], v[48]);
  const float2 d5 = psub(v[5], v[48]);
  const float2 s6 = padd(v[6], v[47]);
  const float2 d6 = psub(v[6], v[47]);
  const float2 s7 = padd(v[7], v[46]);
  const float2 d7 = psub(v[7], v[46]);
  const float2 s8 = padd(v[8], v[45]);
  const float2 d8 = psub(v[8], v[45]);
  const float2 s9 = padd(v[9], v[44]);
  const float2 d9 = psub(v[9], v[44]);
  const float2 s10 = padd(v[10], v[43]);
  const float2 d10 = psub(v[10], v[43]);
  const float2 s11 = padd(v[11], v[42]);
  const float2 d11 = psub(v[11], v[42]);
  const float2 s12 = padd(v[12], v[41]);
  const float2 d12 = psub(v[12], v[41]);
  const float2 s13 = padd(v[13], v[40]);
  const float2 d13 = psub(v[13], v[40]);
  const float2 s14 = padd(v[14], v[39]);
  const float2 d14 = psub(v[14], v[39]);
  const float2 s15 = padd(v[15], v[38]);
  const float2 d15 = psub(v[15], v[38]);
  const float2 s16 = padd(v[16], v[37]);
  const float2 d16 = psub(v[16], v[37]);
  const float2 s17 = padd(v[17], v[36]);
  const float2 d17 = psub(v[17], v[36]);
  const float2 s18 = padd(v[18], v[35]);
  const float2 d18 = psub(v[18], v[35]);
  const float2 s19 = padd(v[19], v[34]);
  const float2 d19 = psub(v[19], v[34]);
  const float2 s20 = padd(v[20], v[33]);
  const float2 d20 = psub(v[20], v[33]);
  const float2 s21 = padd(v[21], v[32]);
  const float2 d21 = psub(v[21], v[32]);
  const float2 s22 = padd(v[22], v[31]);
  const float2 d22 = psub(v[22], v[31]);
  const float2 s23 = padd(v[23], v[30]);
  const float2 d23 = psub(v[23], v[30]);
  const float2 s24 = padd(v[24], v[29]);
  const float2 d24 = psub(v[24], v[29]);
  const float2 s25 = padd(v[25], v[28]);
  const float2 d25 = psub(v[25], v[28]);
  const float2 s26 = padd(v[26], v[27]);
  const float2 d26 = psub(v[26], v[27]);
  if (part == 0) st(0, make_float2(x0.x + (s1.x + s2.x + s3.x + s4.x + s5.x + s6.x + s7.x + s8.x + s9.x + s10.x + s11.x + s12.x + s13.x + s14.x + s15.x + s16.x + s17.x + s18.x + s19.x + s20.x + s21.x + s22.x + s23.x + s24.x + s25.x + s26.x), x0.y + (s1.y + s2.y + s3.y + s4.y + s5.y + s6.y + s7.y + s8.y + s9.y + s10.y + s11.y + s12.y + s13.y + s14.y + s15.y + s16.y + s17.y + s18.y + s19.y + s20.y + s21.y + s22.y + s23.y + s24.y + s25.y + s26.y)));
  switch (part) {
  case 0: {
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.9929810762405396f, ar); ai = fmaf(s1.y, 0.9929810762405396f, ai); br = fmaf(d1.x, 0.11827316880226135f, br); bi = fmaf(d1.y, 0.11827316880226135f, bi);
      ar = fmaf(s2.x, 0.9720228910446167f, ar); ai = fmaf(s2.y, 0.9720228910446167f, ai); br = fmaf(d2.x, 0.2348860502243042f, br); bi = fmaf(d2.y, 0.2348860502243042f, bi);
      ar = fmaf(s3.x, 0.9374196529388428f, ar); ai = fmaf(s3.y, 0.9374196529388428f, ai); br = fmaf(d3.x, 0.3482016324996948f, br); bi = fmaf(d3.y, 0.3482016324996948f, bi);
      ar = fmaf(s4.x, 0.8896570801734924f, ar); ai = fmaf(s4.y, 0.8896570801734924f, ai); br = fmaf(d4.x, 0.4566292464733124f, br); bi = fmaf(d4.y, 0.4566292464733124f, bi);
      ar = fmaf(s5.x, 0.829405665397644f, ar); ai = fmaf(s5.y, 0.829405665397644f, ai); br = fmaf(d5.x, 0.5586467385292053f, br); bi = fmaf(d5.y, 0.5586467385292053f, bi);
      ar = fmaf(s6.x, 0.7575112581253052f, ar); ai = fmaf(s6.y, 0.7575112581253052f, ai); br = fmaf(d6.x, 0.6528221368789673f, br); bi = fmaf(d6.y, 0.6528221368789673f, bi);
      ar = fmaf(s7.x, 0.674983024597168f, ar); ai = fmaf(s7.y, 0.674983024597168f, ai); br = fmaf(d7.x, 0.7378332614898682f, br); bi = fmaf(d7.y, 0.7378332614898682f, bi);
      ar = fmaf(s8.x, 0.5829795002937317f, ar); ai = fmaf(s8.y, 0.5829795002937317f, ai); br = fmaf(d8.x, 0.8124868869781494f, br); bi = fmaf(d8.y, 0.8124868869781494f, bi);
      ar = fmaf(s9.x, 0.4827921986579895f, ar); ai = fmaf(s9.y, 0.4827921986579895f, ai); br = fmaf(d9.x, 0.8757349252700806f, br); bi = fmaf(d9.y, 0.8757349252700806f, bi);
      ar = fmaf(s10.x, 0.3758275806903839f, ar); ai = fmaf(s10.y, 0.3758275806903839f, ai); br = fmaf(d10.x, 0.926689624786377f, br); bi = fmaf(d10.y, 0.926689624786377f, bi);
      ar = fmaf(s11.x, 0.26358717679977417f, ar); ai = fmaf(s11.y, 0.26358717679977417f, ai); br = fmaf(d11.x, 0.9646356105804443f, br); bi = fmaf(d11.y, 0.9646356105804443f, bi);
      ar = fmaf(s12.x, 0.14764656126499176f, ar); ai = fmaf(s12.y, 0.14764656126499176f, ai); br = fmaf(d12.x, 0.989040195941925f, br); bi = fmaf(d12.y, 0.989040195941925f, bi);
      ar = fmaf(s13.x, 0.029633328318595886f, ar); ai = fmaf(s13.y, 0.029633328318595886f, ai); br = fmaf(d13.x, 0.9995608329772949f, br); bi = fmaf(d13.y, 0.9995608329772949f, bi);
      ar = fmaf(s14.x, -0.08879589289426804f, ar); ai = fmaf(s14.y, -0.08879589289426804f, ai); br = fmaf(d14.x, 0.9960498213768005f, br); bi = fmaf(d14.y, 0.9960498213768005f, bi);
      ar = fmaf(s15.x, -0.2059786170721054f, ar); ai = fmaf(s15.y, -0.2059786170721054f, ai); br = fmaf(d15.x, 0.9785565137863159f, br); bi = fmaf(d15.y, 0.9785565137863159f, bi);
      ar = fmaf(s16.x, -0.3202698528766632f, ar); ai = fmaf(s16.y, -0.3202698528766632f, ai); br = fmaf(d16.x, 0.9473263621330261f, br); bi = fmaf(d16.y, 0.9473263621330261f, bi);
      ar = fmaf(s17.x, -0.43006521463394165f, ar); ai = fmaf(s17.y, -0.43006521463394165f, ai); br = fmaf(d17.x, 0.9027978181838989f, br); bi = fmaf(d17.y, 0.9027978181838989f, bi);
      ar = fmaf(s18.x, -0.5338233709335327f, ar); ai = fmaf(s18.y, -0.5338233709335327f, ai); br = fmaf(d18.x, 0.8455960154533386f, br); bi = fmaf(d18.y, 0.8455960154533386f, bi);
      ar = fmaf(s19.x, -0.6300878524780273f, ar); ai = fmaf(s19.y, -0.6300878524780273f, ai); br = fmaf(d19.x, 0.7765238881111145f, br); bi = fmaf(d19.y, 0.7765238881111145f, bi);
      ar = fmaf(s20.x, -0.7175072431564331f, ar); ai = fmaf(s20.y, -0.7175072431564331f, ai); br = fmaf(d20.x, 0.6965510249137878f, br); bi = fmaf(d20.y, 0.6965510249137878f, bi);
      ar = fmaf(s21.x, -0.794854462146759f, ar); ai = fmaf(s21.y, -0.794854462146759f, ai); br = fmaf(d21.x, 0.6068001389503479f, br); bi = fmaf(d21.y, 0.6068001389503479f, bi);
      ar = fmaf(s22.x, -0.8610436320304871f, ar); ai = fmaf(s22.y, -0.8610436320304871f, ai); br = fmaf(d22.x, 0.5085310935974121f, br); bi = fmaf(d22.y, 0.5085310935974121f, bi);
      ar = fmaf(s23.x, -0.9151456356048584f, ar); ai = fmaf(s23.y, -0.9151456356048584f, ai); br = fmaf(d23.x, 0.4031234383583069f, br); bi = fmaf(d23.y, 0.4031234383583069f, bi);
      ar = fmaf(s24.x, -0.956400990486145f, ar); ai = fmaf(s24.y, -0.956400990486145f, ai); br = fmaf(d24.x, 0.29205676913261414f, br); bi = fmaf(d24.y, 0.29205676913261414f, bi);
      ar = fmaf(s25.x, -0.9842305779457092f, ar); ai = fmaf(s25.y, -0.9842305779457092f, ai); br = fmaf(d25.x, 0.1768902689218521f, br); bi = fmaf(d25.y, 0.1768902689218521f, bi);
      ar = fmaf(s26.x, -0.9982437491416931f, ar); ai = fmaf(s26.y, -0.9982437491416931f, ai); br = fmaf(d26.x, 0.05924062803387642f, br); bi = fmaf(d26.y, 0.05924062803387642f, bi);
      if (!INV) { st(1, make_float2(ar + bi, ai - br)); st(52, make_float2(ar - bi, ai + br)); }
      else { st(1, make_float2(ar - bi, ai + br)); st(52, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.9720228910446167f, ar); ai = fmaf(s1.y, 0.9720228910446167f, ai); br = fmaf(d1.x, 0.2348860502243042f, br); bi = fmaf(d1.y, 0.2348860502243042f, bi);
      ar = fmaf(s2.x, 0.8896570801734924f, ar); ai = fmaf(s2.y, 0.8896570801734924f, ai); br = fmaf(d2.x, 0.4566292464733124f, br); bi = fmaf(d2.y, 0.4566292464733124f, bi);
      ar = fmaf(s3.x, 0.7575112581253052f, ar); ai = fmaf(s3.y, 0.7575112581253052f, ai); br = fmaf(d3.x, 0.6528221368789673f, br); bi = fmaf(d3.y, 0.6528221368789673f, bi);
      ar = fmaf(s4.x, 0.5829795002937317f, ar); ai = fmaf(s4.y, 0.5829795002937317f, ai); br = fmaf(d4.x, 0.8124868869781494f, br); bi = fmaf(d4.y, 0.8124868869781494f, bi);
      ar = fmaf(s5.x, 0.3758275806903839f, ar); ai = fmaf(s5.y, 0.3758275806903839f, ai); br = fmaf(d5.x, 0.926689624786377f, br); bi = fmaf(d5.y, 0.926689624786377f, bi);
      ar = fmaf(s6.x, 0.14764656126499176f, ar); ai = fmaf(s6.y, 0.14764656126499176f, ai); br = fmaf(d6.x, 0.989040195941925f, br); bi = fmaf(d6.y, 0.989040195941925f, bi);
      ar = fmaf(s7.x, -0.08879589289426804f, ar); ai = fmaf(s7.y, -0.08879589289426804f, ai); br = fmaf(d7.x, 0.9960498213768005f, br); bi = fmaf(d7.y, 0.9960498213768005f, bi);
      ar = fmaf(s8.x, -0.3202698528766632f, ar); ai = fmaf(s8.y, -0.3202698528766632f, ai); br = fmaf(d8.x, 0.9473263621330261f, br); bi = fmaf(d8.y, 0.9473263621330261f, bi);
      ar = fmaf(s9.x, -0.5338233709335327f, ar); ai = fmaf(s9.y, -0.5338233709335327f, ai); br = fmaf(d9.x, 0.8455960154533386f, br); bi = fmaf(d9.y, 0.8455960154533386f, bi);
      ar = fmaf(s10.x, -0.7175072431564331f, ar); ai = fmaf(s10.y, -0.7175072431564331f, ai); br = fmaf(d10.x, 0.6965510249137878f, br); bi = fmaf(d10.y, 0.6965510249137878f, bi);
      ar = fmaf(s11.x, -0.8610436320304871f, ar); ai = fmaf(s11.y, -0.8610436320304871f, ai); br = fmaf(d11.x, 0.5085310935974121f, br); bi = fmaf(d11.y, 0.5085310935974121f, bi);
      ar = fmaf(s12.x, -0.956400990486145f, ar); ai = fmaf(s12.y, -0.956400990486145f, ai); br = fmaf(d12.x, 0.29205676913261414f, br); bi = fmaf(d12.y, 0.29205676913261414f, bi);
      ar = fmaf(s13.x, -0.9982437491416931f, ar); ai = fmaf(s13.y, -0.9982437491416931f, ai); br = fmaf(d13.x, 0.05924062803387642f, br); bi = fmaf(d13.y, 0.05924062803387642f, bi);
      ar = fmaf(s14.x, -0.9842305779457092f, ar); ai = fmaf(s14.y, -0.9842305779457092f, ai); br = fmaf(d14.x, -0.1768902689218521f, br); bi = fmaf(d14.y, -0.1768902689218521f, bi);
      ar = fmaf(s15.x, -0.9151456356048584f, ar); ai = fmaf(s15.y, -0.9151456356048584f, ai); br = fmaf(d15.x, -0.4031234383583069f, br); bi = fmaf(d15.y, -0.4031234383583069f, bi);
      ar = fmaf(s16.x, -0.794854462146759f, ar); ai = fmaf(s16.y, -0.794854462146759f, ai); br = fmaf(d16.x, -0.6068001389503479f, br); bi = fmaf(d16.y, -0.6068001389503479f, bi);
      ar = fmaf(s17.x, -0.6300878524780273f, ar); ai = fmaf(s17.y, -0.6300878524780273f, ai); br = fmaf(d17.x, -0.7765238881111145f, br); bi = fmaf(d17.y, -0.7765238881111145f, bi);
      ar = fmaf(s18.x, -0.43006521463394165f, ar); ai = fmaf(s18.y, -0.43006521463394165f, ai); br = fmaf(d18.x, -0.9027978181838989f, br); bi = fmaf(d18.y, -0.9027978181838989f, bi);
      ar = fmaf(s19.x, -0.2059786170721054f, ar); ai = fmaf(s19.y, -0.2059786170721054f, ai); br = fmaf(d19.x, -0.9785565137863159f, br); bi = fmaf(d19.y, -0.9785565137863159f, bi);
      ar = fmaf(s20.x, 0.029633328318595886f, ar); ai = fmaf(s20.y, 0.029633328318595886f, ai); br = fmaf(d20.x, -0.9995608329772949f, br); bi = fmaf(d20.y, -0.9995608329772949f, bi);
      ar = fmaf(s21.x, 0.26358717679977417f, ar); ai = fmaf(s21.y, 0.26358717679977417f, ai); br = fmaf(d21.x, -0.9646356105804443f, br); bi = fmaf(d21.y, -0.9646356105804443f, bi);
      ar = fmaf(s22.x, 0.4827921986579895f, ar); ai = fmaf(s22.y, 0.4827921986579895f, ai); br = fmaf(d22.x, -0.8757349252700806f, br); bi = fmaf(d22.y, -0.8757349252700806f, bi);
      ar = fmaf(s23.x, 0.674983024597168f, ar); ai = fmaf(s23.y, 0.674983024597168f, ai); br = fmaf(d23.x, -0.7378332614898682f, br); bi = fmaf(d23.y, -0.7378332614898682f, bi);
      ar = fmaf(s24.x, 0.829405665397644f, ar); ai = fmaf(s24.y, 0.829405665397644f, ai); br = fmaf(d24.x, -0.5586467385292053f, br); bi = fmaf(d24.y, -0.5586467385292053f, bi);
      ar = fmaf(s25.x, 0.9374196529388428f, ar); ai = fmaf(s25.y, 0.9374196529388428f, ai); br = fmaf(d25.x, -0.3482016324996948f, br); bi = fmaf(d25.y, -0.3482016324996948f, bi);
      ar = fmaf(s26.x, 0.9929810762405396f, ar); ai = fmaf(s26.y, 0.9929810762405396f, ai); br = fmaf(d26.x, -0.11827316880226135f, br); bi = fmaf(d26.y, -0.11827316880226135f, bi);
      if (!INV) { st(2, make_float2(ar + bi, ai - br)); st(51, make_float2(ar - bi, ai + br)); }
      else { st(2, make_float2(ar - bi, ai + br)); st(51, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.9374196529388428f, ar); ai = fmaf(s1.y, 0.9374196529388428f, ai); br = fmaf(d1.x, 0.3482016324996948f, br); bi = fmaf(d1.y, 0.3482016324996948f, bi);
      ar = fmaf(s2.x, 0.7575112581253052f, ar); ai = fmaf(s2.y, 0.7575112581253052f, ai); br = fmaf(d2.x, 0.6528221368789673f, br); bi = fmaf(d2.y, 0.6528221368789673f, bi);
      ar = fmaf(s3.x, 0.4827921986579895f, ar); ai = fmaf(s3.y, 0.4827921986579895f, ai); br = fmaf(d3.x, 0.8757349252700806f, br); bi = fmaf(d3.y, 0.8757349252700806f, bi);
      ar = fmaf(s4.x, 0.14764656126499176f, ar); ai = fmaf(s4.y, 0.14764656126499176f, ai); br = fmaf(d4.x, 0.989040195941925f, br); bi = fmaf(d4.y, 0.989040195941925f, bi);
      ar = fmaf(s5.x, -0.2059786170721054f, ar); ai = fmaf(s5.y, -0.2059786170721054f, ai); br = fmaf(d5.x, 0.9785565137863159f, br); bi = fmaf(d5.y, 0.9785565137863159f, bi);
      ar = fmaf(s6.x, -0.5338233709335327f, ar); ai = fmaf(s6.y, -0.5338233709335327f, ai); br = fmaf(d6.x, 0.8455960154533386f, br); bi = fmaf(d6.y, 0.8455960154533386f, bi);
      ar = fmaf(s7.x, -0.794854462146759f, ar); ai = fmaf(s7.y, -0.794854462146759f, ai); br = fmaf(d7.x, 0.6068001389503479f, br); bi = fmaf(d7.y, 0.6068001389503479f, bi);
      ar = fmaf(s8.x, -0.956400990486145f, ar); ai = fmaf(s8.y, -0.956400990486145f, ai); br = fmaf(d8.x, 0.29205676913261414f, br); bi = fmaf(d8.y, 0.29205676913261414f, bi);
      ar = fmaf(s9.x, -0.9982437491416931f, ar); ai = fmaf(s9.y, -0.9982437491416931f, ai); br = fmaf(d9.x, -0.05924062803387642f, br); bi = fmaf(d9.y, -0.05924062803387642f, bi);
      ar = fmaf(s10.x, -0.9151456356048584f, ar); ai = fmaf(s10.y, -0.9151456356048584f, ai); br = fmaf(d10.x, -0.4031234383583069f, br); bi = fmaf(d10.y, -0.4031234383583069f, bi);
      ar = fmaf(s11.x, -0.7175072431564331f, ar); ai = fmaf(s11.y, -0.7175072431564331f, ai); br = fmaf(d11.x, -0.6965510249137878f, br); bi = fmaf(d11.y, -0.6965510249137878f, bi);
      ar = fmaf(s12.x, -0.43006521463394165f, ar); ai = fmaf(s12.y, -0.43006521463394165f, ai); br = fmaf(d12.x, -0.9027978181838989f, br); bi = fmaf(d12.y, -0.9027978181838989f, bi);
      ar = fmaf(s13.x, -0.08879589289426804f, ar); ai = fmaf(s13.y, -0.08879589289426804f, ai); br = fmaf(d13.x, -0.9960498213768005f, br); bi = fmaf(d13.y, -0.9960498213768005f, bi);
      ar = fmaf(s14.x, 0.26358717679977417f, ar); ai = fmaf(s14.y, 0.26358717679977417f, ai); br = fmaf(d14.x, -0.9646356105804443f, br); bi = fmaf(d14.y, -0.9646356105804443f, bi);
      ar = fmaf(s15.x, 0.5829795002937317f, ar); ai = fmaf(s15.y, 0.5829795002937317f, ai); br = fmaf(d15.x, -0.8124868869781494f, br); bi = fmaf(d15.y, -0.8124868869781494f, bi);
      ar = fmaf(s16.x, 0.829405665397644f, ar); ai = fmaf(s16.y, 0.829405665397644f, ai); br = fmaf(d16.x, -0.5586467385292053f, br); bi = fmaf(d16.y, -0.5586467385292053f, bi);
      ar = fmaf(s17.x, 0.9720228910446167f, ar); ai = fmaf(s17.y, 0.9720228910446167f, ai); br = fmaf(d17.x, -0.2348860502243042f, br); bi = fmaf(d17.y, -0.2348860502243042f, bi);
      ar = fmaf(s18.x, 0.9929810762405396f, ar); ai = fmaf(s18.y, 0.9929810762405396f, ai); br = fmaf(d18.x, 0.11827316880226135f, br); bi = fmaf(d18.y, 0.11827316880226135f, bi);
      ar = fmaf(s19.x, 0.8896570801734924f, ar); ai = fmaf(s19.y, 0.8896570801734924f, ai); br = fmaf(d19.x, 0.4566292464733124f, br); bi = fmaf(d19.y, 0.4566292464733124f, bi);
      ar = fmaf(s20.x, 0.674983024597168f, ar); ai = fmaf(s20.y, 0.674983024597168f, ai); br = fmaf(d20.x, 0.7378332614898682f, br); bi = fmaf(d20.y, 0.7378332614898682f, bi);
      ar = fmaf(s21.x, 0.3758275806903839f, ar); ai = fmaf(s21.y, 0.3758275806903839f, ai); br = fmaf(d21.x, 0.926689624786377f, br); bi = fmaf(d21.y, 0.926689624786377f, bi);
      ar = fmaf(s22.x, 0.029633328318595886f, ar); ai = fmaf(s22.y, 0.029633328318595886f, ai); br = fmaf(d22.x, 0.9995608329772949f, br); bi = fmaf(d22.y, 0.9995608329772949f, bi);
      ar = fmaf(s23.x, -0.3202698528766632f, ar); ai = fmaf(s23.y, -0.3202698528766632f, ai); br = fmaf(d23.x, 0.9473263621330261f, br); bi = fmaf(d23.y, 0.9473263621330261f, bi);
      ar = fmaf(s24.x, -0.6300878524780273f, ar); ai = fmaf(s24.y, -0.6300878524780273f, ai); br = fmaf(d24.x, 0.7765238881111145f, br); bi = fmaf(d24.y, 0.7765238881111145f, bi);
      ar = fmaf(s25.x, -0.8610436320304871f, ar); ai = fmaf(s25.y, -0.8610436320304871f, ai); br = fmaf(d25.x, 0.5085310935974121f, br); bi = fmaf(d25.y, 0.5085310935974121f, bi);
      ar = fmaf(s26.x, -0.9842305779457092f, ar); ai = fmaf(s26.y, -0.9842305779457092f, ai); br = fmaf(d26.x, 0.1768902689218521f, br); bi = fmaf(d26.y, 0.1768902689218521f, bi);
      if (!INV) { st(3, make_float2(ar + bi, ai - br)); st(50, make_float2(ar - bi, ai + br)); }
      else { st(3, make_float2(ar - bi, ai + br)); st(50, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.8896570801734924f, ar); ai = fmaf(s1.y, 0.8896570801734924f, ai); br = fmaf(d1.x, 0.4566292464733124f, br); bi = fmaf(d1.y, 0.4566292464733124f, bi);
      ar = fmaf(s2.x, 0.5829795002937317f, ar); ai = fmaf(s2.y, 0.5829795002937317f, ai); br = fmaf(d2.x, 0.8124868869781494f, br); bi = fmaf(d2.y, 0.8124868869781494f, bi);
      ar = fmaf(s3.x, 0.14764656126499176f, ar); ai = fmaf(s3.y, 0.14764656126499176f, ai); br = fmaf(d3.x, 0.989040195941925f, br); bi = fmaf(d3.y, 0.989040195941925f, bi);
      ar = fmaf(s4.x, -0.3202698528766632f, ar); ai = fmaf(s4.y, -0.3202698528766632f, ai); br = fmaf(d4.x, 0.9473263621330261f, br); bi = fmaf(d4.y, 0.9473263621330261f, bi);
      ar = fmaf(s5.x, -0.7175072431564331f, ar); ai = fmaf(s5.y, -0.7175072431564331f, ai); br = fmaf(d5.x, 0.6965510249137878f, br); bi = fmaf(d5.y, 0.6965510249137878f, bi);
      ar = fmaf(s6.x, -0.956400990486145f, ar); ai = fmaf(s6.y, -0.956400990486145f, ai); br = fmaf(d6.x, 0.29205676913261414f, br); bi = fmaf(d6.y, 0.29205676913261414f, bi);
      ar = fmaf(s7.x, -0.9842305779457092f, ar); ai = fmaf(s7.y, -0.9842305779457092f, ai); br = fmaf(d7.x, -0.1768902689218521f, br); bi = fmaf(d7.y, -0.1768902689218521f, bi);
      ar = fmaf(s8.x, -0.794854462146759f, ar); ai = fmaf(s8.y, -0.794854462146759f, ai); br = fmaf(d8.x, -0.6068001389503479f, br); bi = fmaf(d8.y, -0.6068001389503479f, bi);
      ar = fmaf(s9.x, -0.43006521463394165f, ar); ai = fmaf(s9.y, -0.43006521463394165f, ai); br = fmaf(d9.x, -0.9027978181838989f, br); bi = fmaf(d9.y, -0.9027978181838989f, bi);
      ar = fmaf(s10.x, 0.029633328318595886f, ar); ai = fmaf(s10.y, 0.029633328318595886f, ai); br = fmaf(d10.x, -0.9995608329772949f, br); bi = fmaf(d10.y, -0.9995608329772949f, bi);
      ar = fmaf(s11.x, 0.4827921986579895f, ar); ai = fmaf(s11.y, 0.4827921986579895f, ai); br = fmaf(d11.x, -0.8757349252700806f, br); bi = fmaf(d11.y, -0.8757349252700806f, bi);
      ar = fmaf(s12.x, 0.829405665397644f, ar); ai = fmaf(s12.y, 0.829405665397644f, ai); br = fmaf(d12.x, -0.5586467385292053f, br); bi = fmaf(d12.y, -0.5586467385292053f, bi);
      ar = fmaf(s13.x, 0.9929810762405396f, ar); ai = fmaf(s13.y, 0.9929810762405396f, ai); br = fmaf(d13.x, -0.11827316880226135f, br); bi = fmaf(d13.y, -0.11827316880226135f, bi);
      ar = fmaf(s14.x, 0.9374196529388428f, ar); ai = fmaf(s14.y, 0.9374196529388428f, ai); br = fmaf(d14.x, 0.3482016324996948f, br); bi = fmaf(d14.y, 0.3482016324996948f, bi);
      ar = fmaf(s15.x, 0.674983024597168f, ar); ai = fmaf(s15.y, 0.674983024597168f, ai); br = fmaf(d15.x, 0.7378332614898682f, br); bi = fmaf(d15.y, 0.7378332614898682f, bi);
      ar = fmaf(s16.x, 0.26358717679977417f, ar); ai = fmaf(s16.y, 0.26358717679977417f, ai); br = fmaf(d16.x, 0.9646356105804443f, br); bi = fmaf(d16.y, 0.9646356105804443f, bi);
      ar = fmaf(s17.x, -0.2059786170721054f, ar); ai = fmaf(s17.y, -0.2059786170721054f, ai); br = fmaf(d17.x, 0.9785565137863159f, br); bi = fmaf(d17.y, 0.9785565137863159f, bi);
      ar = fmaf(s18.x, -0.6300878524780273f, ar); ai = fmaf(s18.y, -0.6300878524780273f, ai); br = fmaf(d18.x, 0.7765238881111145f, br); bi = fmaf(d18.y, 0.7765238881111145f, bi);
      ar = fmaf(s19.x, -0.9151456356048584f, ar); ai = fmaf(s19.y, -0.9151456356048584f, ai); br = fmaf(d19.x, 0.4031234383583069f, br); bi = fmaf(d19.y, 0.4031234383583069f, bi);
      ar = fmaf(s20.x, -0.9982437491416931f, ar); ai = fmaf(s20.y, -0.9982437491416931f, ai); br = fmaf(d20.x, -0.05924062803387642f, br); bi = fmaf(d20.y, -0.05924062803387642f, bi);
      ar = fmaf(s21.x, -0.8610436320304871f, ar); ai = fmaf(s21.y, -0.8610436320304871f, ai); br = fmaf(d21.x, -0.5085310935974121f, br); bi = fmaf(d21.y, -0.5085310935974121f, bi);
      ar = fmaf(s22.x, -0.5338233709335327f, ar); ai = fmaf(s22.y, -0.5338233709335327f, ai); br = fmaf(d22.x, -0.8455960154533386f, br); bi = fmaf(d22.y, -0.8455960154533386f, bi);
      ar = fmaf(s23.x, -0.08879589289426804f, ar); ai = fmaf(s23.y, -0.08879589289426804f, ai); br = fmaf(d23.x, -0.9960498213768005f, br); bi = fmaf(d23.y, -0.9960498213768005f, bi);
      ar = fmaf(s24.x, 0.3758275806903839f, ar); ai = fmaf(s24.y, 0.3758275806903839f, ai); br = fmaf(d24.x, -0.926689624786377f, br); bi = fmaf(d24.y, -0.926689624786377f, bi);
      ar = fmaf(s25.x, 0.7575112581253052f, ar); ai = fmaf(s25.y, 0.7575112581253052f, ai); br = fmaf(d25.x, -0.6528221368789673f, br); bi = fmaf(d25.y, -0.6528221368789673f, bi);
      ar = fmaf(s26.x, 0.9720228910446167f, ar); ai = fmaf(s26.y, 0.9720228910446167f, ai); br = fmaf(d26.x, -0.2348860502243042f, br); bi = fmaf(d26.y, -0.2348860502243042f, bi);
      if (!INV) { st(4, make_float2(ar + bi, ai - br)); st(49, make_float2(ar - bi, ai + br)); }
      else { st(4, make_float2(ar - bi, ai + br)); st(49, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.829405665397644f, ar); ai = fmaf(s1.y, 0.829405665397644f, ai); br = fmaf(d1.x, 0.5586467385292053f, br); bi = fmaf(d1.y, 0.5586467385292053f, bi);
      ar = fmaf(s2.x, 0.3758275806903839f, ar); ai = fmaf(s2.y, 0.3758275806903839f, ai); br = fmaf(d2.x, 0.926689624786377f, br); bi = fmaf(d2.y, 0.926689624786377f, bi);
      ar = fmaf(s3.x, -0.2059786170721054f, ar); ai = fmaf(s3.y, -0.2059786170721054f, ai); br = fmaf(d3.x, 0.9785565137863159f, br); bi = fmaf(d3.y, 0.9785565137863159f, bi);
      ar = fmaf(s4.x, -0.7175072431564331f, ar); ai = fmaf(s4.y, -0.7175072431564331f, ai); br = fmaf(d4.x, 0.6965510249137878f, br); bi = fmaf(d4.y, 0.6965510249137878f, bi);
      ar = fmaf(s5.x, -0.9842305779457092f, ar); ai = fmaf(s5.y, -0.9842305779457092f, ai); br = fmaf(d5.x, 0.1768902689218521f, br); bi = fmaf(d5.y, 0.1768902689218521f, bi);
      ar = fmaf(s6.x, -0.9151456356048584f, ar); ai = fmaf(s6.y, -0.9151456356048584f, ai); br = fmaf(d6.x, -0.4031234383583069f, br); bi = fmaf(d6.y, -0.4031234383583069f, bi);
      ar = fmaf(s7.x, -0.5338233709335327f, ar); ai = fmaf(s7.y, -0.5338233709335327f, ai); br = fmaf(d7.x, -0.8455960154533386f, br); bi = fmaf(d7.y, -0.8455960154533386f, bi);
      ar = fmaf(s8.x, 0.029633328318595886f, ar); ai = fmaf(s8.y, 0.029633328318595886f, ai); br = fmaf(d8.x, -0.9995608329772949f, br); bi = fmaf(d8.y, -0.9995608329772949f, bi);
      ar = fmaf(s9.x, 0.5829795002937317f, ar); ai = fmaf(s9.y, 0.5829795002937317f, ai); br = fmaf(d9.x, -0.8124868869781494f, br); bi = fmaf(d9.y, -0.8124868869781494f, bi);
      ar = fmaf(s10.x, 0.9374196529388428f, ar); ai = fmaf(s10.y, 0.9374196529388428f, ai); br = fmaf(d10.x, -0.3482016324996948f, br); bi = fmaf(d10.y, -0.3482016324996948f, bi);
      ar = fmaf(s11.x, 0.9720228910446167f, ar); ai = fmaf(s11.y, 0.9720228910446167f, ai); br = fmaf(d11.x, 0.2348860502243042f, br); bi = fmaf(d11.y, 0.2348860502243042f, bi);
      ar = fmaf(s12.x, 0.674983024597168f, ar); ai = fmaf(s12.y, 0.674983024597168f, ai); br = fmaf(d12.x, 0.7378332614898682f, br); bi = fmaf(d12.y, 0.7378332614898682f, bi);
      ar = fmaf(s13.x, 0.14764656126499176f, ar); ai = fmaf(s13.y, 0.14764656126499176f, ai); br = fmaf(d13.x, 0.989040195941925f, br); bi = fmaf(d13.y, 0.989040195941925f, bi);
      ar = fmaf(s14.x, -0.43006521463394165f, ar); ai = fmaf(s14.y, -0.43006521463394165f, ai); br = fmaf(d14.x, 0.9027978181838989f, br); bi = fmaf(d14.y, 0.9027978181838989f, bi);
      ar = fmaf(s15.x, -0.8610436320304871f, ar); ai = fmaf(s15.y, -0.8610436320304871f, ai); br = fmaf(d15.x, 0.5085310935974121f, br); bi = fmaf(d15.y, 0.5085310935974121f, bi);
      ar = fmaf(s16.x, -0.9982437491416931f, ar); ai = fmaf(s16.y, -0.9982437491416931f, ai); br = fmaf(d16.x, -0.05924062803387642f, br); bi = fmaf(d16.y, -0.05924062803387642f, bi);
      ar = fmaf(s17.x, -0.794854462146759f, ar); ai = fmaf(s17.y, -0.794854462146759f, ai); br = fmaf(d17.x, -0.6068001389503479f, br); bi = fmaf(d17.y, -0.6068001389503479f, bi);
      ar = fmaf(s18.x, -0.3202698528766632f, ar); ai = fmaf(s18.y, -0.3202698528766632f, ai); br = fmaf(d18.x, -0.9473263621330261f, br); bi = fmaf(d18.y, -0.9473263621330261f, bi);
      ar = fmaf(s19.x, 0.26358717679977417f, ar); ai = fmaf(s19.y, 0.26358717679977417f, ai); br = fmaf(d19.x, -0.9646356105804443f, br); bi = fmaf(d19.y, -0.9646356105804443f, bi);
      ar = fmaf(s20.x, 0.7575112581253052f, ar); ai = fmaf(s20.y, 0.7575112581253052f, ai); br = fmaf(d20.x, -0.6528221368789673f, br); bi = fmaf(d20.y, -0.6528221368789673f, bi);
      ar = fmaf(s21.x, 0.9929810762405396f, ar); ai = fmaf(s21.y, 0.9929810762405396f, ai); br = fmaf(d21.x, -0.11827316880226135f, br); bi = fmaf(d21.y, -0.11827316880226135f, bi);
      ar = fmaf(s22.x, 0.8896570801734924f, ar); ai = fmaf(s22.y, 0.8896570801734924f, ai); br = fmaf(d22.x, 0.4566292464733124f, br); bi = fmaf(d22.y, 0.4566292464733124f, bi);
      ar = fmaf(s23.x, 0.4827921986579895f, ar); ai = fmaf(s23.y, 0.4827921986579895f, ai); br = fmaf(d23.x, 0.8757349252700806f, br); bi = fmaf(d23.y, 0.8757349252700806f, bi);
      ar = fmaf(s24.x, -0.08879589289426804f, ar); ai = fmaf(s24.y, -0.08879589289426804f, ai); br = fmaf(d24.x, 0.9960498213768005f, br); bi = fmaf(d24.y, 0.9960498213768005f, bi);
      ar = fmaf(s25.x, -0.6300878524780273f, ar); ai = fmaf(s25.y, -0.6300878524780273f, ai); br = fmaf(d25.x, 0.7765238881111145f, br); bi = fmaf(d25.y, 0.7765238881111145f, bi);
      ar = fmaf(s26.x, -0.956400990486145f, ar); ai = fmaf(s26.y, -0.956400990486145f, ai); br = fmaf(d26.x, 0.29205676913261414f, br); bi = fmaf(d26.y, 0.29205676913261414f, bi);
      if (!INV) { st(5, make_float2(ar + bi, ai - br)); st(48, make_float2(ar - bi, ai + br)); }
      else { st(5, make_float2(ar - bi, ai + br)); st(48, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.7575112581253052f, ar); ai = fmaf(s1.y, 0.7575112581253052f, ai); br = fmaf(d1.x, 0.6528221368789673f, br); bi = fmaf(d1.y, 0.6528221368789673f, bi);
      ar = fmaf(s2.x, 0.14764656126499176f, ar); ai = fmaf(s2.y, 0.14764656126499176f, ai); br = fmaf(d2.x, 0.989040195941925f, br); bi = fmaf(d2.y, 0.989040195941925f, bi);
      ar = fmaf(s3.x, -0.5338233709335327f, ar); ai = fmaf(s3.y, -0.5338233709335327f, ai); br = fmaf(d3.x, 0.8455960154533386f, br); bi = fmaf(d3.y, 0.8455960154533386f, bi);
      ar = fmaf(s4.x, -0.956400990486145f, ar); ai = fmaf(s4.y, -0.956400990486145f, ai); br = fmaf(d4.x, 0.29205676913261414f, br); bi = fmaf(d4.y, 0.29205676913261414f, bi);
      ar = fmaf(s5.x, -0.9151456356048584f, ar); ai = fmaf(s5.y, -0.9151456356048584f, ai); br = fmaf(d5.x, -0.4031234383583069f, br); bi = fmaf(d5.y, -0.4031234383583069f, bi);
      ar = fmaf(s6.x, -0.43006521463394165f, ar); ai = fmaf(s6.y, -0.43006521463394165f, ai); br = fmaf(d6.x, -0.9027978181838989f, br); bi = fmaf(d6.y, -0.9027978181838989f, bi);
      ar = fmaf(s7.x, 0.26358717679977417f, ar); ai = fmaf(s7.y, 0.26358717679977417f, ai); br = fmaf(d7.x, -0.9646356105804443f, br); bi = fmaf(d7.y, -0.9646356105804443f, bi);
      ar = fmaf(s8.x, 0.829405665397644f, ar); ai = fmaf(s8.y, 0.829405665397644f, ai); br = fmaf(d8.x, -0.5586467385292053f, br); bi = fmaf(d8.y, -0.5586467385292053f, bi);
      ar = fmaf(s9.x, 0.9929810762405396f, ar); ai = fmaf(s9.y, 0.9929810762405396f, ai); br = fmaf(d9.x, 0.11827316880226135f, br); bi = fmaf(d9.y, 0.11827316880226135f, bi);
      ar = fmaf(s10.x, 0.674983024597168f, ar); ai = fmaf(s10.y, 0.674983024597168f, ai); br = fmaf(d10.x, 0.7378332614898682f, br); bi = fmaf(d10.y, 0.7378332614898682f, bi);
      ar = fmaf(s11.x, 0.029633328318595886f, ar); ai = fmaf(s11.y, 0.029633328318595886f, ai); br = fmaf(d11.x, 0.9995608329772949f, br); bi = fmaf(d11.y, 0.9995608329772949f, bi);
      ar = fmaf(s12.x, -0.6300878524780273f, ar); ai = fmaf(s12.y, -0.6300878524780273f, ai); br = fmaf(d12.x, 0.7765238881111145f, br); bi = fmaf(d12.y, 0.7765238881111145f, bi);
      ar = fmaf(s13.x, -0.9842305779457092f, ar); ai = fmaf(s13.y, -0.9842305779457092f, ai); br = fmaf(d13.x, 0.1768902689218521f, br); bi = fmaf(d13.y, 0.1768902689218521f, bi);
      ar = fmaf(s14.x, -0.8610436320304871f, ar); ai = fmaf(s14.y, -0.8610436320304871f, ai); br = fmaf(d14.x, -0.5085310935974121f, br); bi = fmaf(d14.y, -0.5085310935974121f, bi);
      ar = fmaf(s15.x, -0.3202698528766632f, ar); ai = fmaf(s15.y, -0.3202698528766632f, ai); br = fmaf(d15.x, -0.9473263621330261f, br); bi = fmaf(d15.y, -0.9473263621330261f, bi);
      ar = fmaf(s16.x, 0.3758275806903839f, ar); ai = fmaf(s16.y, 0.3758275806903839f, ai); br = fmaf(d16.x, -0.926689624786377f, br); bi = fmaf(d16.y, -0.926689624786377f, bi);
      ar = fmaf(s17.x, 0.8896570801734924f, ar); ai = fmaf(s17.y, 0.8896570801734924f, ai); br = fmaf(d17.x, -0.4566292464733124f, br); bi = fmaf(d17.y, -0.4566292464733124f, bi);
      ar = fmaf(s18.x, 0.9720228910446167f, ar); ai = fmaf(s18.y, 0.9720228910446167f, ai); br = fmaf(d18.x, 0.2348860502243042f, br); bi = fmaf(d18.y, 0.2348860502243042f, bi);
      ar = fmaf(s19.x, 0.5829795002937317f, ar); ai = fmaf(s19.y, 0.5829795002937317f, ai); br = fmaf(d19.x, 0.8124868869781494f, br); bi = fmaf(d19.y, 0.8124868869781494f, bi);
      ar = fmaf(s20.x, -0.08879589289426804f, ar); ai = fmaf(s20.y, -0.08879589289426804f, ai); br = fmaf(d20.x, 0.9960498213768005f, br); bi = fmaf(d20.y, 0.9960498213768005f, bi);
      ar = fmaf(s21.x, -0.7175072431564331f, ar); ai = fmaf(s21.y, -0.7175072431564331f, ai); br = fmaf(d21.x, 0.6965510249137878f, br); bi = fmaf(d21.y, 0.6965510249137878f, bi);
      ar = fmaf(s22.x, -0.9982437491416931f, ar); ai = fmaf(s22.y, -0.9982437491416931f, ai); br = fmaf(d22.x, 0.05924062803387642f, br); bi = fmaf(d22.y, 0.05924062803387642f, bi);
      ar = fmaf(s23.x, -0.794854462146759f, ar); ai = fmaf(s23.y, -0.794854462146759f, ai); br = fmaf(d23.x, -0.6068001389503479f, br); bi = fmaf(d23.y, -0.6068001389503479f, bi);
      ar = fmaf(s24.x, -0.2059786170721054f, ar); ai = fmaf(s24.y, -0.2059786170721054f, ai); br = fmaf(d24.x, -0.9785565137863159f, br); bi = fmaf(d24.y, -0.9785565137863159f, bi);
      ar = fmaf(s25.x, 0.4827921986579895f, ar); ai = fmaf(s25.y, 0.4827921986579895f, ai); br = fmaf(d25.x, -0.8757349252700806f, br); bi = fmaf(d25.y, -0.8757349252700806f, bi);
      ar = fmaf(s26.x, 0.9374196529388428f, ar); ai = fmaf(s26.y, 0.9374196529388428f, ai); br = fmaf(d26.x, -0.3482016324996948f, br); bi = fmaf(d26.y, -0.3482016324996948f, bi);
      if (!INV) { st(6, make_float2(ar + bi, ai - br)); st(47, make_float2(ar - bi, ai + br)); }
      else { st(6, make_float2(ar - bi, ai + br)); st(47, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.674983024597168f, ar); ai = fmaf(s1.y, 0.674983024597168f, ai); br = fmaf(d1.x, 0.7378332614898682f, br); bi = fmaf(d1.y, 0.7378332614898682f, bi);
      ar = fmaf(s2.x, -0.08879589289426804f, ar); ai = fmaf(s2.y, -0.08879589289426804f, ai); br = fmaf(d2.x, 0.9960498213768005f, br); bi = fmaf(d2.y, 0.9960498213768005f, bi);
      ar = fmaf(s3.x, -0.794854462146759f, ar); ai = fmaf(s3.y, -0.794854462146759f, ai); br = fmaf(d3.x, 0.6068001389503479f, br); bi = fmaf(d3.y, 0.6068001389503479f, bi);
      ar = fmaf(s4.x, -0.9842305779457092f, ar); ai = fmaf(s4.y, -0.9842305779457092f, ai); br = fmaf(d4.x, -0.1768902689218521f, br); bi = fmaf(d4.y, -0.1768902689218521f, bi);
      ar = fmaf(s5.x, -0.5338233709335327f, ar); ai = fmaf(s5.y, -0.5338233709335327f, ai); br = fmaf(d5.x, -0.8455960154533386f, br); bi = fmaf(d5.y, -0.8455960154533386f, bi);
      ar = fmaf(s6.x, 0.26358717679977417f, ar); ai = fmaf(s6.y, 0.26358717679977417f, ai); br = fmaf(d6.x, -0.9646356105804443f, br); bi = fmaf(d6.y, -0.9646356105804443f, bi);
      ar = fmaf(s7.x, 0.8896570801734924f, ar); ai = fmaf(s7.y, 0.8896570801734924f, ai); br = fmaf(d7.x, -0.4566292464733124f, br); bi = fmaf(d7.y, -0.4566292464733124f, bi);
      ar = fmaf(s8.x, 0.9374196529388428f, ar); ai = fmaf(s8.y, 0.9374196529388428f, ai); br = fmaf(d8.x, 0.3482016324996948f, br); bi = fmaf(d8.y, 0.3482016324996948f, bi);
      ar = fmaf(s9.x, 0.3758275806903839f, ar); ai = fmaf(s9.y, 0.3758275806903839f, ai); br = fmaf(d9.x, 0.926689624786377f, br); bi = fmaf(d9.y, 0.926689624786377f, bi);
      ar = fmaf(s10.x, -0.43006521463394165f, ar); ai = fmaf(s10.y, -0.43006521463394165f, ai); br = fmaf(d10.x, 0.9027978181838989f, br); bi = fmaf(d10.y, 0.9027978181838989f, bi);
      ar = fmaf(s11.x, -0.956400990486145f, ar); ai = fmaf(s11.y, -0.956400990486145f, ai); br = fmaf(d11.x, 0.29205676913261414f, br); bi = fmaf(d11.y, 0.29205676913261414f, bi);
      ar = fmaf(s12.x, -0.8610436320304871f, ar); ai = fmaf(s12.y, -0.8610436320304871f, ai); br = fmaf(d12.x, -0.5085310935974121f, br); bi = fmaf(d12.y, -0.5085310935974121f, bi);
      ar = fmaf(s13.x, -0.2059786170721054f, ar); ai = fmaf(s13.y, -0.2059786170721054f, ai); br = fmaf(d13.x, -0.9785565137863159f, br); bi = fmaf(d13.y, -0.9785565137863159f, bi);
      ar = fmaf(s14.x, 0.5829795002937317f, ar); ai = fmaf(s14.y, 0.5829795002937317f, ai); br = fmaf(d14.x, -0.8124868869781494f, br); bi = fmaf(d14.y, -0.8124868869781494f, bi);
      ar = fmaf(s15.x, 0.9929810762405396f, ar); ai = fmaf(s15.y, 0.9929810762405396f, ai); br = fmaf(d15.x, -0.11827316880226135f, br); bi = fmaf(d15.y, -0.11827316880226135f, bi);
      ar = fmaf(s16.x, 0.7575112581253052f, ar); ai = fmaf(s16.y, 0.7575112581253052f, ai); br = fmaf(d16.x, 0.6528221368789673f, br); bi = fmaf(d16.y, 0.6528221368789673f, bi);
      ar = fmaf(s17.x, 0.029633328318595886f, ar); ai = fmaf(s17.y, 0.029633328318595886f, ai); br = fmaf(d17.x, 0.9995608329772949f, br); bi = fmaf(d17.y, 0.9995608329772949f, bi);
      ar = fmaf(s18.x, -0.7175072431564331f, ar); ai = fmaf(s18.y, -0.7175072431564331f, ai); br = fmaf(d18.x, 0.6965510249137878f, br); bi = fmaf(d18.y, 0.6965510249137878f, bi);
      ar = fmaf(s19.x, -0.9982437491416931f, ar); ai = fmaf(s19.y, -0.9982437491416931f, ai); br = fmaf(d19.x, -0.05924062803387642f, br); bi = fmaf(d19.y, -0.05924062803387642f, bi);
      ar = fmaf(s20.x, -0.6300878524780273f, ar); ai = fmaf(s20.y, -0.6300878524780273f, ai); br = fmaf(d20.x, -0.7765238881111145f, br); bi = fmaf(d20.y, -0.7765238881111145f, bi);
      ar = fmaf(s21.x, 0.14764656126499176f, ar); ai = fmaf(s21.y, 0.14764656126499176f, ai); br = fmaf(d21.x, -0.989040195941925f, br); bi = fmaf(d21.y, -0.989040195941925f, bi);
      ar = fmaf(s22.x, 0.829405665397644f, ar); ai = fmaf(s22.y, 0.829405665397644f, ai); br = fmaf(d22.x, -0.5586467385292053f, br); bi = fmaf(d22.y, -0.5586467385292053f, bi);
      ar = fmaf(s23.x, 0.9720228910446167f, ar); ai = fmaf(s23.y, 0.9720228910446167f, ai); br = fmaf(d23.x, 0.2348860502243042f, br); bi = fmaf(d23.y, 0.2348860502243042f, bi);
      ar = fmaf(s24.x, 0.4827921986579895f, ar); ai = fmaf(s24.y, 0.4827921986579895f, ai); br = fmaf(d24.x, 0.8757349252700806f, br); bi = fmaf(d24.y, 0.8757349252700806f, bi);
      ar = fmaf(s25.x, -0.3202698528766632f, ar); ai = fmaf(s25.y, -0.3202698528766632f, ai); br = fmaf(d25.x, 0.9473263621330261f, br); bi = fmaf(d25.y, 0.9473263621330261f, bi);
      ar = fmaf(s26.x, -0.9151456356048584f, ar); ai = fmaf(s26.y, -0.9151456356048584f, ai); br = fmaf(d26.x, 0.4031234383583069f, br); bi = fmaf(d26.y, 0.4031234383583069f, bi);
      if (!INV) { st(7, make_float2(ar + bi, ai - br)); st(46, make_float2(ar - bi, ai + br)); }
      else { st(7, make_float2(ar - bi, ai + br)); st(46, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.5829795002937317f, ar); ai = fmaf(s1.y, 0.5829795002937317f, ai); br = fmaf(d1.x, 0.8124868869781494f, br); bi = fmaf(d1.y, 0.8124868869781494f, bi);
      ar = fmaf(s2.x, -0.3202698528766632f, ar); ai = fmaf(s2.y, -0.3202698528766632f, ai); br = fmaf(d2.x, 0.9473263621330261f, br); bi = fmaf(d2.y, 0.9473263621330261f, bi);
      ar = fmaf(s3.x, -0.956400990486145f, ar); ai = fmaf(s3.y, -0.956400990486145f, ai); br = fmaf(d3.x, 0.29205676913261414f, br); bi = fmaf(d3.y, 0.29205676913261414f, bi);
      ar = fmaf(s4.x, -0.794854462146759f, ar); ai = fmaf(s4.y, -0.794854462146759f, ai); br = fmaf(d4.x, -0.6068001389503479f, br); bi = fmaf(d4.y, -0.6068001389503479f, bi);
      ar = fmaf(s5.x, 0.029633328318595886f, ar); ai = fmaf(s5.y, 0.029633328318595886f, ai); br = fmaf(d5.x, -0.9995608329772949f, br); bi = fmaf(d5.y, -0.9995608329772949f, bi);
      ar = fmaf(s6.x, 0.829405665397644f, ar); ai = fmaf(s6.y, 0.829405665397644f, ai); br = fmaf(d6.x, -0.5586467385292053f, br); bi = fmaf(d6.y, -0.5586467385292053f, bi);
      ar = fmaf(s7.x, 0.9374196529388428f, ar); ai = fmaf(s7.y, 0.9374196529388428f, ai); br = fmaf(d7.x, 0.3482016324996948f, br); bi = fmaf(d7.y, 0.3482016324996948f, bi);
      ar = fmaf(s8.x, 0.26358717679977417f, ar); ai = fmaf(s8.y, 0.26358717679977417f, ai); br = fmaf(d8.x, 0.9646356105804443f, br); bi = fmaf(d8.y, 0.9646356105804443f, bi);
      ar = fmaf(s9.x, -0.6300878524780273f, ar); ai = fmaf(s9.y, -0.6300878524780273f, ai); br = fmaf(d9.x, 0.7765238881111145f, br); bi = fmaf(d9.y, 0.7765238881111145f, bi);
      ar = fmaf(s10.x, -0.9982437491416931f, ar); ai = fmaf(s10.y, -0.9982437491416931f, ai); br = fmaf(d10.x, -0.05924062803387642f, br); bi = fmaf(d10.y, -0.05924062803387642f, bi);
      ar = fmaf(s11.x, -0.5338233709335327f, ar); ai = fmaf(s11.y, -0.5338233709335327f, ai); br = fmaf(d11.x, -0.8455960154533386f, br); bi = fmaf(d11.y, -0.8455960154533386f, bi);
      ar = fmaf(s12.x, 0.3758275806903839f, ar); ai = fmaf(s12.y, 0.3758275806903839f, ai); br = fmaf(d12.x, -0.926689624786377f, br); bi = fmaf(d12.y, -0.926689624786377f, bi);
      ar = fmaf(s13.x, 0.9720228910446167f, ar); ai = fmaf(s13.y, 0.9720228910446167f, ai); br = fmaf(d13.x, -0.2348860502243042f, br); bi = fmaf(d13.y, -0.2348860502243042f, bi);
      ar = fmaf(s14.x, 0.7575112581253052f, ar); ai = fmaf(s14.y, 0.7575112581253052f, ai); br = fmaf(d14.x, 0.6528221368789673f, br); bi = fmaf(d14.y, 0.6528221368789673f, bi);
      ar = fmaf(s15.x, -0.08879589289426804f, ar); ai = fmaf(s15.y, -0.08879589289426804f, ai); br = fmaf(d15.x, 0.9960498213768005f, br); bi = fmaf(d15.y, 0.9960498213768005f, bi);
      ar = fmaf(s16.x, -0.8610436320304871f, ar); ai = fmaf(s16.y, -0.8610436320304871f, ai); br = fmaf(d16.x, 0.5085310935974121f, br); bi = fmaf(d16.y, 0.5085310935974121f, bi);
      ar = fmaf(s17.x, -0.9151456356048584f, ar); ai = fmaf(s17.y, -0.9151456356048584f, ai); br = fmaf(d17.x, -0.4031234383583069f, br); bi = fmaf(d17.y, -0.4031234383583069f, bi);
      ar = fmaf(s18.x, -0.2059786170721054f, ar); ai = fmaf(s18.y, -0.2059786170721054f, ai); br = fmaf(d18.x, -0.9785565137863159f, br); bi = fmaf(d18.y, -0.9785565137863159f, bi);
      ar = fmaf(s19.x, 0.674983024597168f, ar); ai = fmaf(s19.y, 0.674983024597168f, ai); br = fmaf(d19.x, -0.7378332614898682f, br); bi = fmaf(d19.y, -0.7378332614898682f, bi);
      ar = fmaf(s20.x, 0.9929810762405396f, ar); ai = fmaf(s20.y, 0.9929810762405396f, ai); br = fmaf(d20.x, 0.11827316880226135f, br); bi = fmaf(d20.y, 0.11827316880226135f, bi);
      ar = fmaf(s21.x, 0.4827921986579895f, ar); ai = fmaf(s21.y, 0.4827921986579895f, ai); br = fmaf(d21.x, 0.8757349252700806f, br); bi = fmaf(d21.y, 0.8757349252700806f, bi);
      ar = fmaf(s22.x, -0.43006521463394165f, ar); ai = fmaf(s22.y, -0.43006521463394165f, ai); br = fmaf(d22.x, 0.9027978181838989f, br); bi = fmaf(d22.y, 0.9027978181838989f, bi);
      ar = fmaf(s23.x, -0.9842305779457092f, ar); ai = fmaf(s23.y, -0.9842305779457092f, ai); br = fmaf(d23.x, 0.1768902689218521f, br); bi = fmaf(d23.y, 0.1768902689218521f, bi);
      ar = fmaf(s24.x, -0.7175072431564331f, ar); ai = fmaf(s24.y, -0.7175072431564331f, ai); br = fmaf(d24.x, -0.6965510249137878f, br); bi = fmaf(d24.y, -0.6965510249137878f, bi);
      ar = fmaf(s25.x, 0.14764656126499176f, ar); ai = fmaf(s25.y, 0.14764656126499176f, ai); br = fmaf(d25.x, -0.989040195941925f, br); bi = fmaf(d25.y, -0.989040195941925f, bi);
      ar = fmaf(s26.x, 0.8896570801734924f, ar); ai = fmaf(s26.y, 0.8896570801734924f, ai); br = fmaf(d26.x, -0.4566292464733124f, br); bi = fmaf(d26.y, -0.4566292464733124f, bi);
      if (!INV) { st(8, make_float2(ar + bi, ai - br)); st(45, make_float2(ar - bi, ai + br)); }
      else { st(8, make_float2(ar - bi, ai + br)); st(45, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.4827921986579895f, ar); ai = fmaf(s1.y, 0.4827921986579895f, ai); br = fmaf(d1.x, 0.8757349252700806f, br); bi = fmaf(d1.y, 0.8757349252700806f, bi);
      ar = fmaf(s2.x, -0.5338233709335327f, ar); ai = fmaf(s2.y, -0.5338233709335327f, ai); br = fmaf(d2.x, 0.8455960154533386f, br); bi = fmaf(d2.y, 0.8455960154533386f, bi);
      ar = fmaf(s3.x, -0.9982437491416931f, ar); ai = fmaf(s3.y, -0.9982437491416931f, ai); br = fmaf(d3.x, -0.05924062803387642f, br); bi = fmaf(d3.y, -0.05924062803387642f, bi);
      ar = fmaf(s4.x, -0.43006521463394165f, ar); ai = fmaf(s4.y, -0.43006521463394165f, ai); br = fmaf(d4.x, -0.9027978181838989f, br); bi = fmaf(d4.y, -0.9027978181838989f, bi);
      ar = fmaf(s5.x, 0.5829795002937317f, ar); ai = fmaf(s5.y, 0.5829795002937317f, ai); br = fmaf(d5.x, -0.8124868869781494f, br); bi = fmaf(d5.y, -0.8124868869781494f, bi);
      ar = fmaf(s6.x, 0.9929810762405396f, ar); ai = fmaf(s6.y, 0.9929810762405396f, ai); br = fmaf(d6.x, 0.11827316880226135f, br); bi = fmaf(d6.y, 0.11827316880226135f, bi);
      ar = fmaf(s7.x, 0.3758275806903839f, ar); ai = fmaf(s7.y, 0.3758275806903839f, ai); br = fmaf(d7.x, 0.926689624786377f, br); bi = fmaf(d7.y, 0.926689624786377f, bi);
      ar = fmaf(s8.x, -0.6300878524780273f, ar); ai = fmaf(s8.y, -0.6300878524780273f, ai); br = fmaf(d8.x, 0.7765238881111145f, br); bi = fmaf(d8.y, 0.7765238881111145f, bi);
      ar = fmaf(s9.x, -0.9842305779457092f, ar); ai = fmaf(s9.y, -0.9842305779457092f, ai); br = fmaf(d9.x, -0.1768902689218521f, br); bi = fmaf(d9.y, -0.1768902689218521f, bi);
      ar = fmaf(s10.x, -0.3202698528766632f, ar); ai = fmaf(s10.y, -0.3202698528766632f, ai); br = fmaf(d10.x, -0.9473263621330261f, br); bi = fmaf(d10.y, -0.9473263621330261f, bi);
      ar = fmaf(s11.x, 0.674983024597168f, ar); ai = fmaf(s11.y, 0.674983024597168f, ai); br = fmaf(d11.x, -0.7378332614898682f, br); bi = fmaf(d11.y, -0.7378332614898682f, bi);
      ar = fmaf(s12.x, 0.9720228910446167f, ar); ai = fmaf(s12.y, 0.9720228910446167f, ai); br = fmaf(d12.x, 0.2348860502243042f, br); bi = fmaf(d12.y, 0.2348860502243042f, bi);
      ar = fmaf(s13.x, 0.26358717679977417f, ar); ai = fmaf(s13.y, 0.26358717679977417f, ai); br = fmaf(d13.x, 0.9646356105804443f, br); bi = fmaf(d13.y, 0.9646356105804443f, bi);
      ar = fmaf(s14.x, -0.7175072431564331f, ar); ai = fmaf(s14.y, -0.7175072431564331f, ai); br = fmaf(d14.x, 0.6965510249137878f, br); bi = fmaf(d14.y, 0.6965510249137878f, bi);
      ar = fmaf(s15.x, -0.956400990486145f, ar); ai = fmaf(s15.y, -0.956400990486145f, ai); br = fmaf(d15.x, -0.29205676913261414f, br); bi = fmaf(d15.y, -0.29205676913261414f, bi);
      ar = fmaf(s16.x, -0.2059786170721054f, ar); ai = fmaf(s16.y, -0.2059786170721054f, ai); br = fmaf(d16.x, -0.9785565137863159f, br); bi = fmaf(d16.y, -0.9785565137863159f, bi);
      ar = fmaf(s17.x, 0.7575112581253052f, ar); ai = fmaf(s17.y, 0.7575112581253052f, ai); br = fmaf(d17.x, -0.6528221368789673f, br); bi = fmaf(d17.y, -0.6528221368789673f, bi);
      ar = fmaf(s18.x, 0.9374196529388428f, ar); ai = fmaf(s18.y, 0.9374196529388428f, ai); br = fmaf(d18.x, 0.3482016324996948f, br); bi = fmaf(d18.y, 0.3482016324996948f, bi);
      ar = fmaf(s19.x, 0.14764656126499176f, ar); ai = fmaf(s19.y, 0.14764656126499176f, ai); br = fmaf(d19.x, 0.989040195941925f, br); bi = fmaf(d19.y, 0.989040195941925f, bi);
      ar = fmaf(s20.x, -0.794854462146759f, ar); ai = fmaf(s20.y, -0.794854462146759f, ai); br = fmaf(d20.x, 0.6068001389503479f, br); bi = fmaf(d20.y, 0.6068001389503479f, bi);
      ar = fmaf(s21.x, -0.9151456356048584f, ar); ai = fmaf(s21.y, -0.9151456356048584f, ai); br = fmaf(d21.x, -0.4031234383583069f, br); bi = fmaf(d21.y, -0.4031234383583069f, bi);
      ar = fmaf(s22.x, -0.08879589289426804f, ar); ai = fmaf(s22.y, -0.08879589289426804f, ai); br = fmaf(d22.x, -0.9960498213768005f, br); bi = fmaf(d22.y, -0.9960498213768005f, bi);
      ar = fmaf(s23.x, 0.829405665397644f, ar); ai = fmaf(s23.y, 0.829405665397644f, ai); br = fmaf(d23.x, -0.5586467385292053f, br); bi = fmaf(d23.y, -0.5586467385292053f, bi);
      ar = fmaf(s24.x, 0.8896570801734924f, ar); ai = fmaf(s24.y, 0.8896570801734924f, ai); br = fmaf(d24.x, 0.4566292464733124f, br); bi = fmaf(d24.y, 0.4566292464733124f, bi);
      ar = fmaf(s25.x, 0.029633328318595886f, ar); ai = fmaf(s25.y, 0.029633328318595886f, ai); br = fmaf(d25.x, 0.9995608329772949f, br); bi = fmaf(d25.y, 0.9995608329772949f, bi);
      ar = fmaf(s26.x, -0.8610436320304871f, ar); ai = fmaf(s26.y, -0.8610436320304871f, ai); br = fmaf(d26.x, 0.5085310935974121f, br); bi = fmaf(d26.y, 0.5085310935974121f, bi);
      if (!INV) { st(9, make_float2(ar + bi, ai - br)); st(44, make_float2(ar - bi, ai + br)); }
      else { st(9, make_float2(ar - bi, ai + br)); st(44, make_float2(ar + bi, ai - br)); }
    }
    break;
  }
  case 1: {
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.3758275806903839f, ar); ai = fmaf(s1.y, 0.3758275806903839f, ai); br = fmaf(d1.x, 0.926689624786377f, br); bi = fmaf(d1.y, 0.926689624786377f, bi);
      ar = fmaf(s2.x, -0.7175072431564331f, ar); ai = fmaf(s2.y, -0.7175072431564331f, ai); br = fmaf(d2.x, 0.6965510249137878f, br); bi = fmaf(d2.y, 0.6965510249137878f, bi);
      ar = fmaf(s3.x, -0.9151456356048584f, ar); ai = fmaf(s3.y, -0.9151456356048584f, ai); br = fmaf(d3.x, -0.4031234383583069f, br); bi = fmaf(d3.y, -0.4031234383583069f, bi);
      ar = fmaf(s4.x, 0.029633328318595886f, ar); ai = fmaf(s4.y, 0.029633328318595886f, ai); br = fmaf(d4.x, -0.9995608329772949f, br); bi = fmaf(d4.y, -0.9995608329772949f, bi);
      ar = fmaf(s5.x, 0.9374196529388428f, ar); ai = fmaf(s5.y, 0.9374196529388428f, ai); br = fmaf(d5.x, -0.3482016324996948f, br); bi = fmaf(d5.y, -0.3482016324996948f, bi);
      ar = fmaf(s6.x, 0.674983024597168f, ar); ai = fmaf(s6.y, 0.674983024597168f, ai); br = fmaf(d6.x, 0.7378332614898682f, br); bi = fmaf(d6.y, 0.7378332614898682f, bi);
      ar = fmaf(s7.x, -0.43006521463394165f, ar); ai = fmaf(s7.y, -0.43006521463394165f, ai); br = fmaf(d7.x, 0.9027978181838989f, br); bi = fmaf(d7.y, 0.9027978181838989f, bi);
      ar = fmaf(s8.x, -0.9982437491416931f, ar); ai = fmaf(s8.y, -0.9982437491416931f, ai); br = fmaf(d8.x, -0.05924062803387642f, br); bi = fmaf(d8.y, -0.05924062803387642f, bi);
      ar = fmaf(s9.x, -0.3202698528766632f, ar); ai = fmaf(s9.y, -0.3202698528766632f, ai); br = fmaf(d9.x, -0.9473263621330261f, br); bi = fmaf(d9.y, -0.9473263621330261f, bi);
      ar = fmaf(s10.x, 0.7575112581253052f, ar); ai = fmaf(s10.y, 0.7575112581253052f, ai); br = fmaf(d10.x, -0.6528221368789673f, br); bi = fmaf(d10.y, -0.6528221368789673f, bi);
      ar = fmaf(s11.x, 0.8896570801734924f, ar); ai = fmaf(s11.y, 0.8896570801734924f, ai); br = fmaf(d11.x, 0.4566292464733124f, br); bi = fmaf(d11.y, 0.4566292464733124f, bi);
      ar = fmaf(s12.x, -0.08879589289426804f, ar); ai = fmaf(s12.y, -0.08879589289426804f, ai); br = fmaf(d12.x, 0.9960498213768005f, br); bi = fmaf(d12.y, 0.9960498213768005f, bi);
      ar = fmaf(s13.x, -0.956400990486145f, ar); ai = fmaf(s13.y, -0.956400990486145f, ai); br = fmaf(d13.x, 0.29205676913261414f, br); bi = fmaf(d13.y, 0.29205676913261414f, bi);
      ar = fmaf(s14.x, -0.6300878524780273f, ar); ai = fmaf(s14.y, -0.6300878524780273f, ai); br = fmaf(d14.x, -0.7765238881111145f, br); bi = fmaf(d14.y, -0.7765238881111145f, bi);
      ar = fmaf(s15.x, 0.4827921986579895f, ar); ai = fmaf(s15.y, 0.4827921986579895f, ai); br = fmaf(d15.x, -0.8757349252700806f, br); bi = fmaf(d15.y, -0.8757349252700806f, bi);
      ar = fmaf(s16.x, 0.9929810762405396f, ar); ai = fmaf(s16.y, 0.9929810762405396f, ai); br = fmaf(d16.x, 0.11827316880226135f, br); bi = fmaf(d16.y, 0.11827316880226135f, bi);
      ar = fmaf(s17.x, 0.26358717679977417f, ar); ai = fmaf(s17.y, 0.26358717679977417f, ai); br = fmaf(d17.x, 0.9646356105804443f, br); bi = fmaf(d17.y, 0.9646356105804443f, bi);
      ar = fmaf(s18.x, -0.794854462146759f, ar); ai = fmaf(s18.y, -0.794854462146759f, ai); br = fmaf(d18.x, 0.6068001389503479f, br); bi = fmaf(d18.y, 0.6068001389503479f, bi);
      ar = fmaf(s19.x, -0.8610436320304871f, ar); ai = fmaf(s19.y, -0.8610436320304871f, ai); br = fmaf(d19.x, -0.5085310935974121f, br); bi = fmaf(d19.y, -0.5085310935974121f, bi);
      ar = fmaf(s20.x, 0.14764656126499176f, ar); ai = fmaf(s20.y, 0.14764656126499176f, ai); br = fmaf(d20.x, -0.989040195941925f, br); bi = fmaf(d20.y, -0.989040195941925f, bi);
      ar = fmaf(s21.x, 0.9720228910446167f, ar); ai = fmaf(s21.y, 0.9720228910446167f, ai); br = fmaf(d21.x, -0.2348860502243042f, br); bi = fmaf(d21.y, -0.2348860502243042f, bi);
      ar = fmaf(s22.x, 0.5829795002937317f, ar); ai = fmaf(s22.y, 0.5829795002937317f, ai); br = fmaf(d22.x, 0.8124868869781494f, br); bi = fmaf(d22.y, 0.8124868869781494f, bi);
      ar = fmaf(s23.x, -0.5338233709335327f, ar); ai = fmaf(s23.y, -0.5338233709335327f, ai); br = fmaf(d23.x, 0.8455960154533386f, br); bi = fmaf(d23.y, 0.8455960154533386f, bi);
      ar = fmaf(s24.x, -0.9842305779457092f, ar); ai = fmaf(s24.y, -0.9842305779457092f, ai); br = fmaf(d24.x, -0.1768902689218521f, br); bi = fmaf(d24.y, -0.1768902689218521f, bi);
      ar = fmaf(s25.x, -0.2059786170721054f, ar); ai = fmaf(s25.y, -0.2059786170721054f, ai); br = fmaf(d25.x, -0.9785565137863159f, br); bi = fmaf(d25.y, -0.9785565137863159f, bi);
      ar = fmaf(s26.x, 0.829405665397644f, ar); ai = fmaf(s26.y, 0.829405665397644f, ai); br = fmaf(d26.x, -0.5586467385292053f, br); bi = fmaf(d26.y, -0.5586467385292053f, bi);
      if (!INV) { st(10, make_float2(ar + bi, ai - br)); st(43, make_float2(ar - bi, ai + br)); }
      else { st(10, make_float2(ar - bi, ai + br)); st(43, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.26358717679977417f, ar); ai = fmaf(s1.y, 0.26358717679977417f, ai); br = fmaf(d1.x, 0.9646356105804443f, br); bi = fmaf(d1.y, 0.9646356105804443f, bi);
      ar = fmaf(s2.x, -0.8610436320304871f, ar); ai = fmaf(s2.y, -0.8610436320304871f, ai); br = fmaf(d2.x, 0.5085310935974121f, br); bi = fmaf(d2.y, 0.5085310935974121f, bi);
      ar = fmaf(s3.x, -0.7175072431564331f, ar); ai = fmaf(s3.y, -0.7175072431564331f, ai); br = fmaf(d3.x, -0.6965510249137878f, br); bi = fmaf(d3.y, -0.6965510249137878f, bi);
      ar = fmaf(s4.x, 0.4827921986579895f, ar); ai = fmaf(s4.y, 0.4827921986579895f, ai); br = fmaf(d4.x, -0.8757349252700806f, br); bi = fmaf(d4.y, -0.8757349252700806f, bi);
      ar = fmaf(s5.x, 0.9720228910446167f, ar); ai = fmaf(s5.y, 0.9720228910446167f, ai); br = fmaf(d5.x, 0.2348860502243042f, br); bi = fmaf(d5.y, 0.2348860502243042f, bi);
      ar = fmaf(s6.x, 0.029633328318595886f, ar); ai = fmaf(s6.y, 0.029633328318595886f, ai); br = fmaf(d6.x, 0.9995608329772949f, br); bi = fmaf(d6.y, 0.9995608329772949f, bi);
      ar = fmaf(s7.x, -0.956400990486145f, ar); ai = fmaf(s7.y, -0.956400990486145f, ai); br = fmaf(d7.x, 0.29205676913261414f, br); bi = fmaf(d7.y, 0.29205676913261414f, bi);
      ar = fmaf(s8.x, -0.5338233709335327f, ar); ai = fmaf(s8.y, -0.5338233709335327f, ai); br = fmaf(d8.x, -0.8455960154533386f, br); bi = fmaf(d8.y, -0.8455960154533386f, bi);
      ar = fmaf(s9.x, 0.674983024597168f, ar); ai = fmaf(s9.y, 0.674983024597168f, ai); br = fmaf(d9.x, -0.7378332614898682f, br); bi = fmaf(d9.y, -0.7378332614898682f, bi);
      ar = fmaf(s10.x, 0.8896570801734924f, ar); ai = fmaf(s10.y, 0.8896570801734924f, ai); br = fmaf(d10.x, 0.4566292464733124f, br); bi = fmaf(d10.y, 0.4566292464733124f, bi);
      ar = fmaf(s11.x, -0.2059786170721054f, ar); ai = fmaf(s11.y, -0.2059786170721054f, ai); br = fmaf(d11.x, 0.9785565137863159f, br); bi = fmaf(d11.y, 0.9785565137863159f, bi);
      ar = fmaf(s12.x, -0.9982437491416931f, ar); ai = fmaf(s12.y, -0.9982437491416931f, ai); br = fmaf(d12.x, 0.05924062803387642f, br); bi = fmaf(d12.y, 0.05924062803387642f, bi);
      ar = fmaf(s13.x, -0.3202698528766632f, ar); ai = fmaf(s13.y, -0.3202698528766632f, ai); br = fmaf(d13.x, -0.9473263621330261f, br); bi = fmaf(d13.y, -0.9473263621330261f, bi);
      ar = fmaf(s14.x, 0.829405665397644f, ar); ai = fmaf(s14.y, 0.829405665397644f, ai); br = fmaf(d14.x, -0.5586467385292053f, br); bi = fmaf(d14.y, -0.5586467385292053f, bi);
      ar = fmaf(s15.x, 0.7575112581253052f, ar); ai = fmaf(s15.y, 0.7575112581253052f, ai); br = fmaf(d15.x, 0.6528221368789673f, br); bi = fmaf(d15.y, 0.6528221368789673f, bi);
      ar = fmaf(s16.x, -0.43006521463394165f, ar); ai = fmaf(s16.y, -0.43006521463394165f, ai); br = fmaf(d16.x, 0.9027978181838989f, br); bi = fmaf(d16.y, 0.9027978181838989f, bi);
      ar = fmaf(s17.x, -0.9842305779457092f, ar); ai = fmaf(s17.y, -0.9842305779457092f, ai); br = fmaf(d17.x, -0.1768902689218521f, br); bi = fmaf(d17.y, -0.1768902689218521f, bi);
      ar = fmaf(s18.x, -0.08879589289426804f, ar); ai = fmaf(s18.y, -0.08879589289426804f, ai); br = fmaf(d18.x, -0.9960498213768005f, br); bi = fmaf(d18.y, -0.9960498213768005f, bi);
      ar = fmaf(s19.x, 0.9374196529388428f, ar); ai = fmaf(s19.y, 0.9374196529388428f, ai); br = fmaf(d19.x, -0.3482016324996948f, br); bi = fmaf(d19.y, -0.3482016324996948f, bi);
      ar = fmaf(s20.x, 0.5829795002937317f, ar); ai = fmaf(s20.y, 0.5829795002937317f, ai); br = fmaf(d20.x, 0.8124868869781494f, br); bi = fmaf(d20.y, 0.8124868869781494f, bi);
      ar = fmaf(s21.x, -0.6300878524780273f, ar); ai = fmaf(s21.y, -0.6300878524780273f, ai); br = fmaf(d21.x, 0.7765238881111145f, br); bi = fmaf(d21.y, 0.7765238881111145f, bi);
      ar = fmaf(s22.x, -0.9151456356048584f, ar); ai = fmaf(s22.y, -0.9151456356048584f, ai); br = fmaf(d22.x, -0.4031234383583069f, br); bi = fmaf(d22.y, -0.4031234383583069f, bi);
      ar = fmaf(s23.x, 0.14764656126499176f, ar); ai = fmaf(s23.y, 0.14764656126499176f, ai); br = fmaf(d23.x, -0.989040195941925f, br); bi = fmaf(d23.y, -0.989040195941925f, bi);
      ar = fmaf(s24.x, 0.9929810762405396f, ar); ai = fmaf(s24.y, 0.9929810762405396f, ai); br = fmaf(d24.x, -0.11827316880226135f, br); bi = fmaf(d24.y, -0.11827316880226135f, bi);
      ar = fmaf(s25.x, 0.3758275806903839f, ar); ai = fmaf(s25.y, 0.3758275806903839f, ai); br = fmaf(d25.x, 0.926689624786377f, br); bi = fmaf(d25.y, 0.926689624786377f, bi);
      ar = fmaf(s26.x, -0.794854462146759f, ar); ai = fmaf(s26.y, -0.794854462146759f, ai); br = fmaf(d26.x, 0.6068001389503479f, br); bi = fmaf(d26.y, 0.6068001389503479f, bi);
      if (!INV) { st(11, make_float2(ar + bi, ai - br)); st(42, make_float2(ar - bi, ai + br)); }
      else { st(11, make_float2(ar - bi, ai + br)); st(42, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.14764656126499176f, ar); ai = fmaf(s1.y, 0.14764656126499176f, ai); br = fmaf(d1.x, 0.989040195941925f, br); bi = fmaf(d1.y, 0.989040195941925f, bi);
      ar = fmaf(s2.x, -0.956400990486145f, ar); ai = fmaf(s2.y, -0.956400990486145f, ai); br = fmaf(d2.x, 0.29205676913261414f, br); bi = fmaf(d2.y, 0.29205676913261414f, bi);
      ar = fmaf(s3.x, -0.43006521463394165f, ar); ai = fmaf(s3.y, -0.43006521463394165f, ai); br = fmaf(d3.x, -0.9027978181838989f, br); bi = fmaf(d3.y, -0.9027978181838989f, bi);
      ar = fmaf(s4.x, 0.829405665397644f, ar); ai = fmaf(s4.y, 0.829405665397644f, ai); br = fmaf(d4.x, -0.5586467385292053f, br); bi = fmaf(d4.y, -0.5586467385292053f, bi);
      ar = fmaf(s5.x, 0.674983024597168f, ar); ai = fmaf(s5.y, 0.674983024597168f, ai); br = fmaf(d5.x, 0.7378332614898682f, br); bi = fmaf(d5.y, 0.7378332614898682f, bi);
      ar = fmaf(s6.x, -0.6300878524780273f, ar); ai = fmaf(s6.y, -0.6300878524780273f, ai); br = fmaf(d6.x, 0.7765238881111145f, br); bi = fmaf(d6.y, 0.7765238881111145f, bi);
      ar = fmaf(s7.x, -0.8610436320304871f, ar); ai = fmaf(s7.y, -0.8610436320304871f, ai); br = fmaf(d7.x, -0.5085310935974121f, br); bi = fmaf(d7.y, -0.5085310935974121f, bi);
      ar = fmaf(s8.x, 0.3758275806903839f, ar); ai = fmaf(s8.y, 0.3758275806903839f, ai); br = fmaf(d8.x, -0.926689624786377f, br); bi = fmaf(d8.y, -0.926689624786377f, bi);
      ar = fmaf(s9.x, 0.9720228910446167f, ar); ai = fmaf(s9.y, 0.9720228910446167f, ai); br = fmaf(d9.x, 0.2348860502243042f, br); bi = fmaf(d9.y, 0.2348860502243042f, bi);
      ar = fmaf(s10.x, -0.08879589289426804f, ar); ai = fmaf(s10.y, -0.08879589289426804f, ai); br = fmaf(d10.x, 0.9960498213768005f, br); bi = fmaf(d10.y, 0.9960498213768005f, bi);
      ar = fmaf(s11.x, -0.9982437491416931f, ar); ai = fmaf(s11.y, -0.9982437491416931f, ai); br = fmaf(d11.x, 0.05924062803387642f, br); bi = fmaf(d11.y, 0.05924062803387642f, bi);
      ar = fmaf(s12.x, -0.2059786170721054f, ar); ai = fmaf(s12.y, -0.2059786170721054f, ai); br = fmaf(d12.x, -0.9785565137863159f, br); bi = fmaf(d12.y, -0.9785565137863159f, bi);
      ar = fmaf(s13.x, 0.9374196529388428f, ar); ai = fmaf(s13.y, 0.9374196529388428f, ai); br = fmaf(d13.x, -0.3482016324996948f, br); bi = fmaf(d13.y, -0.3482016324996948f, bi);
      ar = fmaf(s14.x, 0.4827921986579895f, ar); ai = fmaf(s14.y, 0.4827921986579895f, ai); br = fmaf(d14.x, 0.8757349252700806f, br); bi = fmaf(d14.y, 0.8757349252700806f, bi);
      ar = fmaf(s15.x, -0.794854462146759f, ar); ai = fmaf(s15.y, -0.794854462146759f, ai); br = fmaf(d15.x, 0.6068001389503479f, br); bi = fmaf(d15.y, 0.6068001389503479f, bi);
      ar = fmaf(s16.x, -0.7175072431564331f, ar); ai = fmaf(s16.y, -0.7175072431564331f, ai); br = fmaf(d16.x, -0.6965510249137878f, br); bi = fmaf(d16.y, -0.6965510249137878f, bi);
      ar = fmaf(s17.x, 0.5829795002937317f, ar); ai = fmaf(s17.y, 0.5829795002937317f, ai); br = fmaf(d17.x, -0.8124868869781494f, br); bi = fmaf(d17.y, -0.8124868869781494f, bi);
      ar = fmaf(s18.x, 0.8896570801734924f, ar); ai = fmaf(s18.y, 0.8896570801734924f, ai); br = fmaf(d18.x, 0.4566292464733124f, br); bi = fmaf(d18.y, 0.4566292464733124f, bi);
      ar = fmaf(s19.x, -0.3202698528766632f, ar); ai = fmaf(s19.y, -0.3202698528766632f, ai); br = fmaf(d19.x, 0.9473263621330261f, br); bi = fmaf(d19.y, 0.9473263621330261f, bi);
      ar = fmaf(s20.x, -0.9842305779457092f, ar); ai = fmaf(s20.y, -0.9842305779457092f, ai); br = fmaf(d20.x, -0.1768902689218521f, br); bi = fmaf(d20.y, -0.1768902689218521f, bi);
      ar = fmaf(s21.x, 0.029633328318595886f, ar); ai = fmaf(s21.y, 0.029633328318595886f, ai); br = fmaf(d21.x, -0.9995608329772949f, br); bi = fmaf(d21.y, -0.9995608329772949f, bi);
      ar = fmaf(s22.x, 0.9929810762405396f, ar); ai = fmaf(s22.y, 0.9929810762405396f, ai); br = fmaf(d22.x, -0.11827316880226135f, br); bi = fmaf(d22.y, -0.11827316880226135f, bi);
      ar = fmaf(s23.x, 0.26358717679977417f, ar); ai = fmaf(s23.y, 0.26358717679977417f, ai); br = fmaf(d23.x, 0.9646356105804443f, br); bi = fmaf(d23.y, 0.9646356105804443f, bi);
      ar = fmaf(s24.x, -0.9151456356048584f, ar); ai = fmaf(s24.y, -0.9151456356048584f, ai); br = fmaf(d24.x, 0.4031234383583069f, br); bi = fmaf(d24.y, 0.4031234383583069f, bi);
      ar = fmaf(s25.x, -0.5338233709335327f, ar); ai = fmaf(s25.y, -0.5338233709335327f, ai); br = fmaf(d25.x, -0.8455960154533386f, br); bi = fmaf(d25.y, -0.8455960154533386f, bi);
      ar = fmaf(s26.x, 0.7575112581253052f, ar); ai = fmaf(s26.y, 0.7575112581253052f, ai); br = fmaf(d26.x, -0.6528221368789673f, br); bi = fmaf(d26.y, -0.6528221368789673f, bi);
      if (!INV) { st(12, make_float2(ar + bi, ai - br)); st(41, make_float2(ar - bi, ai + br)); }
      else { st(12, make_float2(ar - bi, ai + br)); st(41, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, 0.029633328318595886f, ar); ai = fmaf(s1.y, 0.029633328318595886f, ai); br = fmaf(d1.x, 0.9995608329772949f, br); bi = fmaf(d1.y, 0.9995608329772949f, bi);
      ar = fmaf(s2.x, -0.9982437491416931f, ar); ai = fmaf(s2.y, -0.9982437491416931f, ai); br = fmaf(d2.x, 0.05924062803387642f, br); bi = fmaf(d2.y, 0.05924062803387642f, bi);
      ar = fmaf(s3.x, -0.08879589289426804f, ar); ai = fmaf(s3.y, -0.08879589289426804f, ai); br = fmaf(d3.x, -0.9960498213768005f, br); bi = fmaf(d3.y, -0.9960498213768005f, bi);
      ar = fmaf(s4.x, 0.9929810762405396f, ar); ai = fmaf(s4.y, 0.9929810762405396f, ai); br = fmaf(d4.x, -0.11827316880226135f, br); bi = fmaf(d4.y, -0.11827316880226135f, bi);
      ar = fmaf(s5.x, 0.14764656126499176f, ar); ai = fmaf(s5.y, 0.14764656126499176f, ai); br = fmaf(d5.x, 0.989040195941925f, br); bi = fmaf(d5.y, 0.989040195941925f, bi);
      ar = fmaf(s6.x, -0.9842305779457092f, ar); ai = fmaf(s6.y, -0.9842305779457092f, ai); br = fmaf(d6.x, 0.1768902689218521f, br); bi = fmaf(d6.y, 0.1768902689218521f, bi);
      ar = fmaf(s7.x, -0.2059786170721054f, ar); ai = fmaf(s7.y, -0.2059786170721054f, ai); br = fmaf(d7.x, -0.9785565137863159f, br); bi = fmaf(d7.y, -0.9785565137863159f, bi);
      ar = fmaf(s8.x, 0.9720228910446167f, ar); ai = fmaf(s8.y, 0.9720228910446167f, ai); br = fmaf(d8.x, -0.2348860502243042f, br); bi = fmaf(d8.y, -0.2348860502243042f, bi);
      ar = fmaf(s9.x, 0.26358717679977417f, ar); ai = fmaf(s9.y, 0.26358717679977417f, ai); br = fmaf(d9.x, 0.9646356105804443f, br); bi = fmaf(d9.y, 0.9646356105804443f, bi);
      ar = fmaf(s10.x, -0.956400990486145f, ar); ai = fmaf(s10.y, -0.956400990486145f, ai); br = fmaf(d10.x, 0.29205676913261414f, br); bi = fmaf(d10.y, 0.29205676913261414f, bi);
      ar = fmaf(s11.x, -0.3202698528766632f, ar); ai = fmaf(s11.y, -0.3202698528766632f, ai); br = fmaf(d11.x, -0.9473263621330261f, br); bi = fmaf(d11.y, -0.9473263621330261f, bi);
      ar = fmaf(s12.x, 0.9374196529388428f, ar); ai = fmaf(s12.y, 0.9374196529388428f, ai); br = fmaf(d12.x, -0.3482016324996948f, br); bi = fmaf(d12.y, -0.3482016324996948f, bi);
      ar = fmaf(s13.x, 0.3758275806903839f, ar); ai = fmaf(s13.y, 0.3758275806903839f, ai); br = fmaf(d13.x, 0.926689624786377f, br); bi = fmaf(d13.y, 0.926689624786377f, bi);
      ar = fmaf(s14.x, -0.9151456356048584f, ar); ai = fmaf(s14.y, -0.9151456356048584f, ai); br = fmaf(d14.x, 0.4031234383583069f, br); bi = fmaf(d14.y, 0.4031234383583069f, bi);
      ar = fmaf(s15.x, -0.43006521463394165f, ar); ai = fmaf(s15.y, -0.43006521463394165f, ai); br = fmaf(d15.x, -0.9027978181838989f, br); bi = fmaf(d15.y, -0.9027978181838989f, bi);
      ar = fmaf(s16.x, 0.8896570801734924f, ar); ai = fmaf(s16.y, 0.8896570801734924f, ai); br = fmaf(d16.x, -0.4566292464733124f, br); bi = fmaf(d16.y, -0.4566292464733124f, bi);
      ar = fmaf(s17.x, 0.4827921986579895f, ar); ai = fmaf(s17.y, 0.4827921986579895f, ai); br = fmaf(d17.x, 0.8757349252700806f, br); bi = fmaf(d17.y, 0.8757349252700806f, bi);
      ar = fmaf(s18.x, -0.8610436320304871f, ar); ai = fmaf(s18.y, -0.8610436320304871f, ai); br = fmaf(d18.x, 0.5085310935974121f, br); bi = fmaf(d18.y, 0.5085310935974121f, bi);
      ar = fmaf(s19.x, -0.5338233709335327f, ar); ai = fmaf(s19.y, -0.5338233709335327f, ai); br = fmaf(d19.x, -0.8455960154533386f, br); bi = fmaf(d19.y, -0.8455960154533386f, bi);
      ar = fmaf(s20.x, 0.829405665397644f, ar); ai = fmaf(s20.y, 0.829405665397644f, ai); br = fmaf(d20.x, -0.5586467385292053f, br); bi = fmaf(d20.y, -0.5586467385292053f, bi);
      ar = fmaf(s21.x, 0.5829795002937317f, ar); ai = fmaf(s21.y, 0.5829795002937317f, ai); br = fmaf(d21.x, 0.8124868869781494f, br); bi = fmaf(d21.y, 0.8124868869781494f, bi);
      ar = fmaf(s22.x, -0.794854462146759f, ar); ai = fmaf(s22.y, -0.794854462146759f, ai); br = fmaf(d22.x, 0.6068001389503479f, br); bi = fmaf(d22.y, 0.6068001389503479f, bi);
      ar = fmaf(s23.x, -0.6300878524780273f, ar); ai = fmaf(s23.y, -0.6300878524780273f, ai); br = fmaf(d23.x, -0.7765238881111145f, br); bi = fmaf(d23.y, -0.7765238881111145f, bi);
      ar = fmaf(s24.x, 0.7575112581253052f, ar); ai = fmaf(s24.y, 0.7575112581253052f, ai); br = fmaf(d24.x, -0.6528221368789673f, br); bi = fmaf(d24.y, -0.6528221368789673f, bi);
      ar = fmaf(s25.x, 0.674983024597168f, ar); ai = fmaf(s25.y, 0.674983024597168f, ai); br = fmaf(d25.x, 0.7378332614898682f, br); bi = fmaf(d25.y, 0.7378332614898682f, bi);
      ar = fmaf(s26.x, -0.7175072431564331f, ar); ai = fmaf(s26.y, -0.7175072431564331f, ai); br = fmaf(d26.x, 0.6965510249137878f, br); bi = fmaf(d26.y, 0.6965510249137878f, bi);
      if (!INV) { st(13, make_float2(ar + bi, ai - br)); st(40, make_float2(ar - bi, ai + br)); }
      else { st(13, make_float2(ar - bi, ai + br)); st(40, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.08879589289426804f, ar); ai = fmaf(s1.y, -0.08879589289426804f, ai); br = fmaf(d1.x, 0.9960498213768005f, br); bi = fmaf(d1.y, 0.9960498213768005f, bi);
      ar = fmaf(s2.x, -0.9842305779457092f, ar); ai = fmaf(s2.y, -0.9842305779457092f, ai); br = fmaf(d2.x, -0.1768902689218521f, br); bi = fmaf(d2.y, -0.1768902689218521f, bi);
      ar = fmaf(s3.x, 0.26358717679977417f, ar); ai = fmaf(s3.y, 0.26358717679977417f, ai); br = fmaf(d3.x, -0.9646356105804443f, br); bi = fmaf(d3.y, -0.9646356105804443f, bi);
      ar = fmaf(s4.x, 0.9374196529388428f, ar); ai = fmaf(s4.y, 0.9374196529388428f, ai); br = fmaf(d4.x, 0.3482016324996948f, br); bi = fmaf(d4.y, 0.3482016324996948f, bi);
      ar = fmaf(s5.x, -0.43006521463394165f, ar); ai = fmaf(s5.y, -0.43006521463394165f, ai); br = fmaf(d5.x, 0.9027978181838989f, br); bi = fmaf(d5.y, 0.9027978181838989f, bi);
      ar = fmaf(s6.x, -0.8610436320304871f, ar); ai = fmaf(s6.y, -0.8610436320304871f, ai); br = fmaf(d6.x, -0.5085310935974121f, br); bi = fmaf(d6.y, -0.5085310935974121f, bi);
      ar = fmaf(s7.x, 0.5829795002937317f, ar); ai = fmaf(s7.y, 0.5829795002937317f, ai); br = fmaf(d7.x, -0.8124868869781494f, br); bi = fmaf(d7.y, -0.8124868869781494f, bi);
      ar = fmaf(s8.x, 0.7575112581253052f, ar); ai = fmaf(s8.y, 0.7575112581253052f, ai); br = fmaf(d8.x, 0.6528221368789673f, br); bi = fmaf(d8.y, 0.6528221368789673f, bi);
      ar = fmaf(s9.x, -0.7175072431564331f, ar); ai = fmaf(s9.y, -0.7175072431564331f, ai); br = fmaf(d9.x, 0.6965510249137878f, br); bi = fmaf(d9.y, 0.6965510249137878f, bi);
      ar = fmaf(s10.x, -0.6300878524780273f, ar); ai = fmaf(s10.y, -0.6300878524780273f, ai); br = fmaf(d10.x, -0.7765238881111145f, br); bi = fmaf(d10.y, -0.7765238881111145f, bi);
      ar = fmaf(s11.x, 0.829405665397644f, ar); ai = fmaf(s11.y, 0.829405665397644f, ai); br = fmaf(d11.x, -0.5586467385292053f, br); bi = fmaf(d11.y, -0.5586467385292053f, bi);
      ar = fmaf(s12.x, 0.4827921986579895f, ar); ai = fmaf(s12.y, 0.4827921986579895f, ai); br = fmaf(d12.x, 0.8757349252700806f, br); bi = fmaf(d12.y, 0.8757349252700806f, bi);
      ar = fmaf(s13.x, -0.9151456356048584f, ar); ai = fmaf(s13.y, -0.9151456356048584f, ai); br = fmaf(d13.x, 0.4031234383583069f, br); bi = fmaf(d13.y, 0.4031234383583069f, bi);
      ar = fmaf(s14.x, -0.3202698528766632f, ar); ai = fmaf(s14.y, -0.3202698528766632f, ai); br = fmaf(d14.x, -0.9473263621330261f, br); bi = fmaf(d14.y, -0.9473263621330261f, bi);
      ar = fmaf(s15.x, 0.9720228910446167f, ar); ai = fmaf(s15.y, 0.9720228910446167f, ai); br = fmaf(d15.x, -0.2348860502243042f, br); bi = fmaf(d15.y, -0.2348860502243042f, bi);
      ar = fmaf(s16.x, 0.14764656126499176f, ar); ai = fmaf(s16.y, 0.14764656126499176f, ai); br = fmaf(d16.x, 0.989040195941925f, br); bi = fmaf(d16.y, 0.989040195941925f, bi);
      ar = fmaf(s17.x, -0.9982437491416931f, ar); ai = fmaf(s17.y, -0.9982437491416931f, ai); br = fmaf(d17.x, 0.05924062803387642f, br); bi = fmaf(d17.y, 0.05924062803387642f, bi);
      ar = fmaf(s18.x, 0.029633328318595886f, ar); ai = fmaf(s18.y, 0.029633328318595886f, ai); br = fmaf(d18.x, -0.9995608329772949f, br); bi = fmaf(d18.y, -0.9995608329772949f, bi);
      ar = fmaf(s19.x, 0.9929810762405396f, ar); ai = fmaf(s19.y, 0.9929810762405396f, ai); br = fmaf(d19.x, 0.11827316880226135f, br); bi = fmaf(d19.y, 0.11827316880226135f, bi);
      ar = fmaf(s20.x, -0.2059786170721054f, ar); ai = fmaf(s20.y, -0.2059786170721054f, ai); br = fmaf(d20.x, 0.9785565137863159f, br); bi = fmaf(d20.y, 0.9785565137863159f, bi);
      ar = fmaf(s21.x, -0.956400990486145f, ar); ai = fmaf(s21.y, -0.956400990486145f, ai); br = fmaf(d21.x, -0.29205676913261414f, br); bi = fmaf(d21.y, -0.29205676913261414f, bi);
      ar = fmaf(s22.x, 0.3758275806903839f, ar); ai = fmaf(s22.y, 0.3758275806903839f, ai); br = fmaf(d22.x, -0.926689624786377f, br); bi = fmaf(d22.y, -0.926689624786377f, bi);
      ar = fmaf(s23.x, 0.8896570801734924f, ar); ai = fmaf(s23.y, 0.8896570801734924f, ai); br = fmaf(d23.x, 0.4566292464733124f, br); bi = fmaf(d23.y, 0.4566292464733124f, bi);
      ar = fmaf(s24.x, -0.5338233709335327f, ar); ai = fmaf(s24.y, -0.5338233709335327f, ai); br = fmaf(d24.x, 0.8455960154533386f, br); bi = fmaf(d24.y, 0.8455960154533386f, bi);
      ar = fmaf(s25.x, -0.794854462146759f, ar); ai = fmaf(s25.y, -0.794854462146759f, ai); br = fmaf(d25.x, -0.6068001389503479f, br); bi = fmaf(d25.y, -0.6068001389503479f, bi);
      ar = fmaf(s26.x, 0.674983024597168f, ar); ai = fmaf(s26.y, 0.674983024597168f, ai); br = fmaf(d26.x, -0.7378332614898682f, br); bi = fmaf(d26.y, -0.7378332614898682f, bi);
      if (!INV) { st(14, make_float2(ar + bi, ai - br)); st(39, make_float2(ar - bi, ai + br)); }
      else { st(14, make_float2(ar - bi, ai + br)); st(39, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.2059786170721054f, ar); ai = fmaf(s1.y, -0.2059786170721054f, ai); br = fmaf(d1.x, 0.9785565137863159f, br); bi = fmaf(d1.y, 0.9785565137863159f, bi);
      ar = fmaf(s2.x, -0.9151456356048584f, ar); ai = fmaf(s2.y, -0.9151456356048584f, ai); br = fmaf(d2.x, -0.4031234383583069f, br); bi = fmaf(d2.y, -0.4031234383583069f, bi);
      ar = fmaf(s3.x, 0.5829795002937317f, ar); ai = fmaf(s3.y, 0.5829795002937317f, ai); br = fmaf(d3.x, -0.8124868869781494f, br); bi = fmaf(d3.y, -0.8124868869781494f, bi);
      ar = fmaf(s4.x, 0.674983024597168f, ar); ai = fmaf(s4.y, 0.674983024597168f, ai); br = fmaf(d4.x, 0.7378332614898682f, br); bi = fmaf(d4.y, 0.7378332614898682f, bi);
      ar = fmaf(s5.x, -0.8610436320304871f, ar); ai = fmaf(s5.y, -0.8610436320304871f, ai); br = fmaf(d5.x, 0.5085310935974121f, br); bi = fmaf(d5.y, 0.5085310935974121f, bi);
      ar = fmaf(s6.x, -0.3202698528766632f, ar); ai = fmaf(s6.y, -0.3202698528766632f, ai); br = fmaf(d6.x, -0.9473263621330261f, br); bi = fmaf(d6.y, -0.9473263621330261f, bi);
      ar = fmaf(s7.x, 0.9929810762405396f, ar); ai = fmaf(s7.y, 0.9929810762405396f, ai); br = fmaf(d7.x, -0.11827316880226135f, br); bi = fmaf(d7.y, -0.11827316880226135f, bi);
      ar = fmaf(s8.x, -0.08879589289426804f, ar); ai = fmaf(s8.y, -0.08879589289426804f, ai); br = fmaf(d8.x, 0.9960498213768005f, br); bi = fmaf(d8.y, 0.9960498213768005f, bi);
      ar = fmaf(s9.x, -0.956400990486145f, ar); ai = fmaf(s9.y, -0.956400990486145f, ai); br = fmaf(d9.x, -0.29205676913261414f, br); bi = fmaf(d9.y, -0.29205676913261414f, bi);
      ar = fmaf(s10.x, 0.4827921986579895f, ar); ai = fmaf(s10.y, 0.4827921986579895f, ai); br = fmaf(d10.x, -0.8757349252700806f, br); bi = fmaf(d10.y, -0.8757349252700806f, bi);
      ar = fmaf(s11.x, 0.7575112581253052f, ar); ai = fmaf(s11.y, 0.7575112581253052f, ai); br = fmaf(d11.x, 0.6528221368789673f, br); bi = fmaf(d11.y, 0.6528221368789673f, bi);
      ar = fmaf(s12.x, -0.794854462146759f, ar); ai = fmaf(s12.y, -0.794854462146759f, ai); br = fmaf(d12.x, 0.6068001389503479f, br); bi = fmaf(d12.y, 0.6068001389503479f, bi);
      ar = fmaf(s13.x, -0.43006521463394165f, ar); ai = fmaf(s13.y, -0.43006521463394165f, ai); br = fmaf(d13.x, -0.9027978181838989f, br); bi = fmaf(d13.y, -0.9027978181838989f, bi);
      ar = fmaf(s14.x, 0.9720228910446167f, ar); ai = fmaf(s14.y, 0.9720228910446167f, ai); br = fmaf(d14.x, -0.2348860502243042f, br); bi = fmaf(d14.y, -0.2348860502243042f, bi);
      ar = fmaf(s15.x, 0.029633328318595886f, ar); ai = fmaf(s15.y, 0.029633328318595886f, ai); br = fmaf(d15.x, 0.9995608329772949f, br); bi = fmaf(d15.y, 0.9995608329772949f, bi);
      ar = fmaf(s16.x, -0.9842305779457092f, ar); ai = fmaf(s16.y, -0.9842305779457092f, ai); br = fmaf(d16.x, -0.1768902689218521f, br); bi = fmaf(d16.y, -0.1768902689218521f, bi);
      ar = fmaf(s17.x, 0.3758275806903839f, ar); ai = fmaf(s17.y, 0.3758275806903839f, ai); br = fmaf(d17.x, -0.926689624786377f, br); bi = fmaf(d17.y, -0.926689624786377f, bi);
      ar = fmaf(s18.x, 0.829405665397644f, ar); ai = fmaf(s18.y, 0.829405665397644f, ai); br = fmaf(d18.x, 0.5586467385292053f, br); bi = fmaf(d18.y, 0.5586467385292053f, bi);
      ar = fmaf(s19.x, -0.7175072431564331f, ar); ai = fmaf(s19.y, -0.7175072431564331f, ai); br = fmaf(d19.x, 0.6965510249137878f, br); bi = fmaf(d19.y, 0.6965510249137878f, bi);
      ar = fmaf(s20.x, -0.5338233709335327f, ar); ai = fmaf(s20.y, -0.5338233709335327f, ai); br = fmaf(d20.x, -0.8455960154533386f, br); bi = fmaf(d20.y, -0.8455960154533386f, bi);
      ar = fmaf(s21.x, 0.9374196529388428f, ar); ai = fmaf(s21.y, 0.9374196529388428f, ai); br = fmaf(d21.x, -0.3482016324996948f, br); bi = fmaf(d21.y, -0.3482016324996948f, bi);
      ar = fmaf(s22.x, 0.14764656126499176f, ar); ai = fmaf(s22.y, 0.14764656126499176f, ai); br = fmaf(d22.x, 0.989040195941925f, br); bi = fmaf(d22.y, 0.989040195941925f, bi);
      ar = fmaf(s23.x, -0.9982437491416931f, ar); ai = fmaf(s23.y, -0.9982437491416931f, ai); br = fmaf(d23.x, -0.05924062803387642f, br); bi = fmaf(d23.y, -0.05924062803387642f, bi);
      ar = fmaf(s24.x, 0.26358717679977417f, ar); ai = fmaf(s24.y, 0.26358717679977417f, ai); br = fmaf(d24.x, -0.9646356105804443f, br); bi = fmaf(d24.y, -0.9646356105804443f, bi);
      ar = fmaf(s25.x, 0.8896570801734924f, ar); ai = fmaf(s25.y, 0.8896570801734924f, ai); br = fmaf(d25.x, 0.4566292464733124f, br); bi = fmaf(d25.y, 0.4566292464733124f, bi);
      ar = fmaf(s26.x, -0.6300878524780273f, ar); ai = fmaf(s26.y, -0.6300878524780273f, ai); br = fmaf(d26.x, 0.7765238881111145f, br); bi = fmaf(d26.y, 0.7765238881111145f, bi);
      if (!INV) { st(15, make_float2(ar + bi, ai - br)); st(38, make_float2(ar - bi, ai + br)); }
      else { st(15, make_float2(ar - bi, ai + br)); st(38, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.3202698528766632f, ar); ai = fmaf(s1.y, -0.3202698528766632f, ai); br = fmaf(d1.x, 0.9473263621330261f, br); bi = fmaf(d1.y, 0.9473263621330261f, bi);
      ar = fmaf(s2.x, -0.794854462146759f, ar); ai = fmaf(s2.y, -0.794854462146759f, ai); br = fmaf(d2.x, -0.6068001389503479f, br); bi = fmaf(d2.y, -0.6068001389503479f, bi);
      ar = fmaf(s3.x, 0.829405665397644f, ar); ai = fmaf(s3.y, 0.829405665397644f, ai); br = fmaf(d3.x, -0.5586467385292053f, br); bi = fmaf(d3.y, -0.5586467385292053f, bi);
      ar = fmaf(s4.x, 0.26358717679977417f, ar); ai = fmaf(s4.y, 0.26358717679977417f, ai); br = fmaf(d4.x, 0.9646356105804443f, br); bi = fmaf(d4.y, 0.9646356105804443f, bi);
      ar = fmaf(s5.x, -0.9982437491416931f, ar); ai = fmaf(s5.y, -0.9982437491416931f, ai); br = fmaf(d5.x, -0.05924062803387642f, br); bi = fmaf(d5.y, -0.05924062803387642f, bi);
      ar = fmaf(s6.x, 0.3758275806903839f, ar); ai = fmaf(s6.y, 0.3758275806903839f, ai); br = fmaf(d6.x, -0.926689624786377f, br); bi = fmaf(d6.y, -0.926689624786377f, bi);
      ar = fmaf(s7.x, 0.7575112581253052f, ar); ai = fmaf(s7.y, 0.7575112581253052f, ai); br = fmaf(d7.x, 0.6528221368789673f, br); bi = fmaf(d7.y, 0.6528221368789673f, bi);
      ar = fmaf(s8.x, -0.8610436320304871f, ar); ai = fmaf(s8.y, -0.8610436320304871f, ai); br = fmaf(d8.x, 0.5085310935974121f, br); bi = fmaf(d8.y, 0.5085310935974121f, bi);
      ar = fmaf(s9.x, -0.2059786170721054f, ar); ai = fmaf(s9.y, -0.2059786170721054f, ai); br = fmaf(d9.x, -0.9785565137863159f, br); bi = fmaf(d9.y, -0.9785565137863159f, bi);
      ar = fmaf(s10.x, 0.9929810762405396f, ar); ai = fmaf(s10.y, 0.9929810762405396f, ai); br = fmaf(d10.x, 0.11827316880226135f, br); bi = fmaf(d10.y, 0.11827316880226135f, bi);
      ar = fmaf(s11.x, -0.43006521463394165f, ar); ai = fmaf(s11.y, -0.43006521463394165f, ai); br = fmaf(d11.x, 0.9027978181838989f, br); bi = fmaf(d11.y, 0.9027978181838989f, bi);
      ar = fmaf(s12.x, -0.7175072431564331f, ar); ai = fmaf(s12.y, -0.7175072431564331f, ai); br = fmaf(d12.x, -0.6965510249137878f, br); bi = fmaf(d12.y, -0.6965510249137878f, bi);
      ar = fmaf(s13.x, 0.8896570801734924f, ar); ai = fmaf(s13.y, 0.8896570801734924f, ai); br = fmaf(d13.x, -0.4566292464733124f, br); bi = fmaf(d13.y, -0.4566292464733124f, bi);
      ar = fmaf(s14.x, 0.14764656126499176f, ar); ai = fmaf(s14.y, 0.14764656126499176f, ai); br = fmaf(d14.x, 0.989040195941925f, br); bi = fmaf(d14.y, 0.989040195941925f, bi);
      ar = fmaf(s15.x, -0.9842305779457092f, ar); ai = fmaf(s15.y, -0.9842305779457092f, ai); br = fmaf(d15.x, -0.1768902689218521f, br); bi = fmaf(d15.y, -0.1768902689218521f, bi);
      ar = fmaf(s16.x, 0.4827921986579895f, ar); ai = fmaf(s16.y, 0.4827921986579895f, ai); br = fmaf(d16.x, -0.8757349252700806f, br); bi = fmaf(d16.y, -0.8757349252700806f, bi);
      ar = fmaf(s17.x, 0.674983024597168f, ar); ai = fmaf(s17.y, 0.674983024597168f, ai); br = fmaf(d17.x, 0.7378332614898682f, br); bi = fmaf(d17.y, 0.7378332614898682f, bi);
      ar = fmaf(s18.x, -0.9151456356048584f, ar); ai = fmaf(s18.y, -0.9151456356048584f, ai); br = fmaf(d18.x, 0.4031234383583069f, br); bi = fmaf(d18.y, 0.4031234383583069f, bi);
      ar = fmaf(s19.x, -0.08879589289426804f, ar); ai = fmaf(s19.y, -0.08879589289426804f, ai); br = fmaf(d19.x, -0.9960498213768005f, br); bi = fmaf(d19.y, -0.9960498213768005f, bi);
      ar = fmaf(s20.x, 0.9720228910446167f, ar); ai = fmaf(s20.y, 0.9720228910446167f, ai); br = fmaf(d20.x, 0.2348860502243042f, br); bi = fmaf(d20.y, 0.2348860502243042f, bi);
      ar = fmaf(s21.x, -0.5338233709335327f, ar); ai = fmaf(s21.y, -0.5338233709335327f, ai); br = fmaf(d21.x, 0.8455960154533386f, br); bi = fmaf(d21.y, 0.8455960154533386f, bi);
      ar = fmaf(s22.x, -0.6300878524780273f, ar); ai = fmaf(s22.y, -0.6300878524780273f, ai); br = fmaf(d22.x, -0.7765238881111145f, br); bi = fmaf(d22.y, -0.7765238881111145f, bi);
      ar = fmaf(s23.x, 0.9374196529388428f, ar); ai = fmaf(s23.y, 0.9374196529388428f, ai); br = fmaf(d23.x, -0.3482016324996948f, br); bi = fmaf(d23.y, -0.3482016324996948f, bi);
      ar = fmaf(s24.x, 0.029633328318595886f, ar); ai = fmaf(s24.y, 0.029633328318595886f, ai); br = fmaf(d24.x, 0.9995608329772949f, br); bi = fmaf(d24.y, 0.9995608329772949f, bi);
      ar = fmaf(s25.x, -0.956400990486145f, ar); ai = fmaf(s25.y, -0.956400990486145f, ai); br = fmaf(d25.x, -0.29205676913261414f, br); bi = fmaf(d25.y, -0.29205676913261414f, bi);
      ar = fmaf(s26.x, 0.5829795002937317f, ar); ai = fmaf(s26.y, 0.5829795002937317f, ai); br = fmaf(d26.x, -0.8124868869781494f, br); bi = fmaf(d26.y, -0.8124868869781494f, bi);
      if (!INV) { st(16, make_float2(ar + bi, ai - br)); st(37, make_float2(ar - bi, ai + br)); }
      else { st(16, make_float2(ar - bi, ai + br)); st(37, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.43006521463394165f, ar); ai = fmaf(s1.y, -0.43006521463394165f, ai); br = fmaf(d1.x, 0.9027978181838989f, br); bi = fmaf(d1.y, 0.9027978181838989f, bi);
      ar = fmaf(s2.x, -0.6300878524780273f, ar); ai = fmaf(s2.y, -0.6300878524780273f, ai); br = fmaf(d2.x, -0.7765238881111145f, br); bi = fmaf(d2.y, -0.7765238881111145f, bi);
      ar = fmaf(s3.x, 0.9720228910446167f, ar); ai = fmaf(s3.y, 0.9720228910446167f, ai); br = fmaf(d3.x, -0.2348860502243042f, br); bi = fmaf(d3.y, -0.2348860502243042f, bi);
      ar = fmaf(s4.x, -0.2059786170721054f, ar); ai = fmaf(s4.y, -0.2059786170721054f, ai); br = fmaf(d4.x, 0.9785565137863159f, br); bi = fmaf(d4.y, 0.9785565137863159f, bi);
      ar = fmaf(s5.x, -0.794854462146759f, ar); ai = fmaf(s5.y, -0.794854462146759f, ai); br = fmaf(d5.x, -0.6068001389503479f, br); bi = fmaf(d5.y, -0.6068001389503479f, bi);
      ar = fmaf(s6.x, 0.8896570801734924f, ar); ai = fmaf(s6.y, 0.8896570801734924f, ai); br = fmaf(d6.x, -0.4566292464733124f, br); bi = fmaf(d6.y, -0.4566292464733124f, bi);
      ar = fmaf(s7.x, 0.029633328318595886f, ar); ai = fmaf(s7.y, 0.029633328318595886f, ai); br = fmaf(d7.x, 0.9995608329772949f, br); bi = fmaf(d7.y, 0.9995608329772949f, bi);
      ar = fmaf(s8.x, -0.9151456356048584f, ar); ai = fmaf(s8.y, -0.9151456356048584f, ai); br = fmaf(d8.x, -0.4031234383583069f, br); bi = fmaf(d8.y, -0.4031234383583069f, bi);
      ar = fmaf(s9.x, 0.7575112581253052f, ar); ai = fmaf(s9.y, 0.7575112581253052f, ai); br = fmaf(d9.x, -0.6528221368789673f, br); bi = fmaf(d9.y, -0.6528221368789673f, bi);
      ar = fmaf(s10.x, 0.26358717679977417f, ar); ai = fmaf(s10.y, 0.26358717679977417f, ai); br = fmaf(d10.x, 0.9646356105804443f, br); bi = fmaf(d10.y, 0.9646356105804443f, bi);
      ar = fmaf(s11.x, -0.9842305779457092f, ar); ai = fmaf(s11.y, -0.9842305779457092f, ai); br = fmaf(d11.x, -0.1768902689218521f, br); bi = fmaf(d11.y, -0.1768902689218521f, bi);
      ar = fmaf(s12.x, 0.5829795002937317f, ar); ai = fmaf(s12.y, 0.5829795002937317f, ai); br = fmaf(d12.x, -0.8124868869781494f, br); bi = fmaf(d12.y, -0.8124868869781494f, bi);
      ar = fmaf(s13.x, 0.4827921986579895f, ar); ai = fmaf(s13.y, 0.4827921986579895f, ai); br = fmaf(d13.x, 0.8757349252700806f, br); bi = fmaf(d13.y, 0.8757349252700806f, bi);
      ar = fmaf(s14.x, -0.9982437491416931f, ar); ai = fmaf(s14.y, -0.9982437491416931f, ai); br = fmaf(d14.x, 0.05924062803387642f, br); bi = fmaf(d14.y, 0.05924062803387642f, bi);
      ar = fmaf(s15.x, 0.3758275806903839f, ar); ai = fmaf(s15.y, 0.3758275806903839f, ai); br = fmaf(d15.x, -0.926689624786377f, br); bi = fmaf(d15.y, -0.926689624786377f, bi);
      ar = fmaf(s16.x, 0.674983024597168f, ar); ai = fmaf(s16.y, 0.674983024597168f, ai); br = fmaf(d16.x, 0.7378332614898682f, br); bi = fmaf(d16.y, 0.7378332614898682f, bi);
      ar = fmaf(s17.x, -0.956400990486145f, ar); ai = fmaf(s17.y, -0.956400990486145f, ai); br = fmaf(d17.x, 0.29205676913261414f, br); bi = fmaf(d17.y, 0.29205676913261414f, bi);
      ar = fmaf(s18.x, 0.14764656126499176f, ar); ai = fmaf(s18.y, 0.14764656126499176f, ai); br = fmaf(d18.x, -0.989040195941925f, br); bi = fmaf(d18.y, -0.989040195941925f, bi);
      ar = fmaf(s19.x, 0.829405665397644f, ar); ai = fmaf(s19.y, 0.829405665397644f, ai); br = fmaf(d19.x, 0.5586467385292053f, br); bi = fmaf(d19.y, 0.5586467385292053f, bi);
      ar = fmaf(s20.x, -0.8610436320304871f, ar); ai = fmaf(s20.y, -0.8610436320304871f, ai); br = fmaf(d20.x, 0.5085310935974121f, br); bi = fmaf(d20.y, 0.5085310935974121f, bi);
      ar = fmaf(s21.x, -0.08879589289426804f, ar); ai = fmaf(s21.y, -0.08879589289426804f, ai); br = fmaf(d21.x, -0.9960498213768005f, br); bi = fmaf(d21.y, -0.9960498213768005f, bi);
      ar = fmaf(s22.x, 0.9374196529388428f, ar); ai = fmaf(s22.y, 0.9374196529388428f, ai); br = fmaf(d22.x, 0.3482016324996948f, br); bi = fmaf(d22.y, 0.3482016324996948f, bi);
      ar = fmaf(s23.x, -0.7175072431564331f, ar); ai = fmaf(s23.y, -0.7175072431564331f, ai); br = fmaf(d23.x, 0.6965510249137878f, br); bi = fmaf(d23.y, 0.6965510249137878f, bi);
      ar = fmaf(s24.x, -0.3202698528766632f, ar); ai = fmaf(s24.y, -0.3202698528766632f, ai); br = fmaf(d24.x, -0.9473263621330261f, br); bi = fmaf(d24.y, -0.9473263621330261f, bi);
      ar = fmaf(s25.x, 0.9929810762405396f, ar); ai = fmaf(s25.y, 0.9929810762405396f, ai); br = fmaf(d25.x, 0.11827316880226135f, br); bi = fmaf(d25.y, 0.11827316880226135f, bi);
      ar = fmaf(s26.x, -0.5338233709335327f, ar); ai = fmaf(s26.y, -0.5338233709335327f, ai); br = fmaf(d26.x, 0.8455960154533386f, br); bi = fmaf(d26.y, 0.8455960154533386f, bi);
      if (!INV) { st(17, make_float2(ar + bi, ai - br)); st(36, make_float2(ar - bi, ai + br)); }
      else { st(17, make_float2(ar - bi, ai + br)); st(36, make_float2(ar + bi, ai - br)); }
    }
    break;
  }
  case 2: {
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.5338233709335327f, ar); ai = fmaf(s1.y, -0.5338233709335327f, ai); br = fmaf(d1.x, 0.8455960154533386f, br); bi = fmaf(d1.y, 0.8455960154533386f, bi);
      ar = fmaf(s2.x, -0.43006521463394165f, ar); ai = fmaf(s2.y, -0.43006521463394165f, ai); br = fmaf(d2.x, -0.9027978181838989f, br); bi = fmaf(d2.y, -0.9027978181838989f, bi);
      ar = fmaf(s3.x, 0.9929810762405396f, ar); ai = fmaf(s3.y, 0.9929810762405396f, ai); br = fmaf(d3.x, 0.11827316880226135f, br); bi = fmaf(d3.y, 0.11827316880226135f, bi);
      ar = fmaf(s4.x, -0.6300878524780273f, ar); ai = fmaf(s4.y, -0.6300878524780273f, ai); br = fmaf(d4.x, 0.7765238881111145f, br); bi = fmaf(d4.y, 0.7765238881111145f, bi);
      ar = fmaf(s5.x, -0.3202698528766632f, ar); ai = fmaf(s5.y, -0.3202698528766632f, ai); br = fmaf(d5.x, -0.9473263621330261f, br); bi = fmaf(d5.y, -0.9473263621330261f, bi);
      ar = fmaf(s6.x, 0.9720228910446167f, ar); ai = fmaf(s6.y, 0.9720228910446167f, ai); br = fmaf(d6.x, 0.2348860502243042f, br); bi = fmaf(d6.y, 0.2348860502243042f, bi);
      ar = fmaf(s7.x, -0.7175072431564331f, ar); ai = fmaf(s7.y, -0.7175072431564331f, ai); br = fmaf(d7.x, 0.6965510249137878f, br); bi = fmaf(d7.y, 0.6965510249137878f, bi);
      ar = fmaf(s8.x, -0.2059786170721054f, ar); ai = fmaf(s8.y, -0.2059786170721054f, ai); br = fmaf(d8.x, -0.9785565137863159f, br); bi = fmaf(d8.y, -0.9785565137863159f, bi);
      ar = fmaf(s9.x, 0.9374196529388428f, ar); ai = fmaf(s9.y, 0.9374196529388428f, ai); br = fmaf(d9.x, 0.3482016324996948f, br); bi = fmaf(d9.y, 0.3482016324996948f, bi);
      ar = fmaf(s10.x, -0.794854462146759f, ar); ai = fmaf(s10.y, -0.794854462146759f, ai); br = fmaf(d10.x, 0.6068001389503479f, br); bi = fmaf(d10.y, 0.6068001389503479f, bi);
      ar = fmaf(s11.x, -0.08879589289426804f, ar); ai = fmaf(s11.y, -0.08879589289426804f, ai); br = fmaf(d11.x, -0.9960498213768005f, br); bi = fmaf(d11.y, -0.9960498213768005f, bi);
      ar = fmaf(s12.x, 0.8896570801734924f, ar); ai = fmaf(s12.y, 0.8896570801734924f, ai); br = fmaf(d12.x, 0.4566292464733124f, br); bi = fmaf(d12.y, 0.4566292464733124f, bi);
      ar = fmaf(s13.x, -0.8610436320304871f, ar); ai = fmaf(s13.y, -0.8610436320304871f, ai); br = fmaf(d13.x, 0.5085310935974121f, br); bi = fmaf(d13.y, 0.5085310935974121f, bi);
      ar = fmaf(s14.x, 0.029633328318595886f, ar); ai = fmaf(s14.y, 0.029633328318595886f, ai); br = fmaf(d14.x, -0.9995608329772949f, br); bi = fmaf(d14.y, -0.9995608329772949f, bi);
      ar = fmaf(s15.x, 0.829405665397644f, ar); ai = fmaf(s15.y, 0.829405665397644f, ai); br = fmaf(d15.x, 0.5586467385292053f, br); bi = fmaf(d15.y, 0.5586467385292053f, bi);
      ar = fmaf(s16.x, -0.9151456356048584f, ar); ai = fmaf(s16.y, -0.9151456356048584f, ai); br = fmaf(d16.x, 0.4031234383583069f, br); bi = fmaf(d16.y, 0.4031234383583069f, bi);
      ar = fmaf(s17.x, 0.14764656126499176f, ar); ai = fmaf(s17.y, 0.14764656126499176f, ai); br = fmaf(d17.x, -0.989040195941925f, br); bi = fmaf(d17.y, -0.989040195941925f, bi);
      ar = fmaf(s18.x, 0.7575112581253052f, ar); ai = fmaf(s18.y, 0.7575112581253052f, ai); br = fmaf(d18.x, 0.6528221368789673f, br); bi = fmaf(d18.y, 0.6528221368789673f, bi);
      ar = fmaf(s19.x, -0.956400990486145f, ar); ai = fmaf(s19.y, -0.956400990486145f, ai); br = fmaf(d19.x, 0.29205676913261414f, br); bi = fmaf(d19.y, 0.29205676913261414f, bi);
      ar = fmaf(s20.x, 0.26358717679977417f, ar); ai = fmaf(s20.y, 0.26358717679977417f, ai); br = fmaf(d20.x, -0.9646356105804443f, br); bi = fmaf(d20.y, -0.9646356105804443f, bi);
      ar = fmaf(s21.x, 0.674983024597168f, ar); ai = fmaf(s21.y, 0.674983024597168f, ai); br = fmaf(d21.x, 0.7378332614898682f, br); bi = fmaf(d21.y, 0.7378332614898682f, bi);
      ar = fmaf(s22.x, -0.9842305779457092f, ar); ai = fmaf(s22.y, -0.9842305779457092f, ai); br = fmaf(d22.x, 0.1768902689218521f, br); bi = fmaf(d22.y, 0.1768902689218521f, bi);
      ar = fmaf(s23.x, 0.3758275806903839f, ar); ai = fmaf(s23.y, 0.3758275806903839f, ai); br = fmaf(d23.x, -0.926689624786377f, br); bi = fmaf(d23.y, -0.926689624786377f, bi);
      ar = fmaf(s24.x, 0.5829795002937317f, ar); ai = fmaf(s24.y, 0.5829795002937317f, ai); br = fmaf(d24.x, 0.8124868869781494f, br); bi = fmaf(d24.y, 0.8124868869781494f, bi);
      ar = fmaf(s25.x, -0.9982437491416931f, ar); ai = fmaf(s25.y, -0.9982437491416931f, ai); br = fmaf(d25.x, 0.05924062803387642f, br); bi = fmaf(d25.y, 0.05924062803387642f, bi);
      ar = fmaf(s26.x, 0.4827921986579895f, ar); ai = fmaf(s26.y, 0.4827921986579895f, ai); br = fmaf(d26.x, -0.8757349252700806f, br); bi = fmaf(d26.y, -0.8757349252700806f, bi);
      if (!INV) { st(18, make_float2(ar + bi, ai - br)); st(35, make_float2(ar - bi, ai + br)); }
      else { st(18, make_float2(ar - bi, ai + br)); st(35, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.6300878524780273f, ar); ai = fmaf(s1.y, -0.6300878524780273f, ai); br = fmaf(d1.x, 0.7765238881111145f, br); bi = fmaf(d1.y, 0.7765238881111145f, bi);
      ar = fmaf(s2.x, -0.2059786170721054f, ar); ai = fmaf(s2.y, -0.2059786170721054f, ai); br = fmaf(d2.x, -0.9785565137863159f, br); bi = fmaf(d2.y, -0.9785565137863159f, bi);
      ar = fmaf(s3.x, 0.8896570801734924f, ar); ai = fmaf(s3.y, 0.8896570801734924f, ai); br = fmaf(d3.x, 0.4566292464733124f, br); bi = fmaf(d3.y, 0.4566292464733124f, bi);
      ar = fmaf(s4.x, -0.9151456356048584f, ar); ai = fmaf(s4.y, -0.9151456356048584f, ai); br = fmaf(d4.x, 0.4031234383583069f, br); bi = fmaf(d4.y, 0.4031234383583069f, bi);
      ar = fmaf(s5.x, 0.26358717679977417f, ar); ai = fmaf(s5.y, 0.26358717679977417f, ai); br = fmaf(d5.x, -0.9646356105804443f, br); bi = fmaf(d5.y, -0.9646356105804443f, bi);
      ar = fmaf(s6.x, 0.5829795002937317f, ar); ai = fmaf(s6.y, 0.5829795002937317f, ai); br = fmaf(d6.x, 0.8124868869781494f, br); bi = fmaf(d6.y, 0.8124868869781494f, bi);
      ar = fmaf(s7.x, -0.9982437491416931f, ar); ai = fmaf(s7.y, -0.9982437491416931f, ai); br = fmaf(d7.x, -0.05924062803387642f, br); bi = fmaf(d7.y, -0.05924062803387642f, bi);
      ar = fmaf(s8.x, 0.674983024597168f, ar); ai = fmaf(s8.y, 0.674983024597168f, ai); br = fmaf(d8.x, -0.7378332614898682f, br); bi = fmaf(d8.y, -0.7378332614898682f, bi);
      ar = fmaf(s9.x, 0.14764656126499176f, ar); ai = fmaf(s9.y, 0.14764656126499176f, ai); br = fmaf(d9.x, 0.989040195941925f, br); bi = fmaf(d9.y, 0.989040195941925f, bi);
      ar = fmaf(s10.x, -0.8610436320304871f, ar); ai = fmaf(s10.y, -0.8610436320304871f, ai); br = fmaf(d10.x, -0.5085310935974121f, br); bi = fmaf(d10.y, -0.5085310935974121f, bi);
      ar = fmaf(s11.x, 0.9374196529388428f, ar); ai = fmaf(s11.y, 0.9374196529388428f, ai); br = fmaf(d11.x, -0.3482016324996948f, br); bi = fmaf(d11.y, -0.3482016324996948f, bi);
      ar = fmaf(s12.x, -0.3202698528766632f, ar); ai = fmaf(s12.y, -0.3202698528766632f, ai); br = fmaf(d12.x, 0.9473263621330261f, br); bi = fmaf(d12.y, 0.9473263621330261f, bi);
      ar = fmaf(s13.x, -0.5338233709335327f, ar); ai = fmaf(s13.y, -0.5338233709335327f, ai); br = fmaf(d13.x, -0.8455960154533386f, br); bi = fmaf(d13.y, -0.8455960154533386f, bi);
      ar = fmaf(s14.x, 0.9929810762405396f, ar); ai = fmaf(s14.y, 0.9929810762405396f, ai); br = fmaf(d14.x, 0.11827316880226135f, br); bi = fmaf(d14.y, 0.11827316880226135f, bi);
      ar = fmaf(s15.x, -0.7175072431564331f, ar); ai = fmaf(s15.y, -0.7175072431564331f, ai); br = fmaf(d15.x, 0.6965510249137878f, br); bi = fmaf(d15.y, 0.6965510249137878f, bi);
      ar = fmaf(s16.x, -0.08879589289426804f, ar); ai = fmaf(s16.y, -0.08879589289426804f, ai); br = fmaf(d16.x, -0.9960498213768005f, br); bi = fmaf(d16.y, -0.9960498213768005f, bi);
      ar = fmaf(s17.x, 0.829405665397644f, ar); ai = fmaf(s17.y, 0.829405665397644f, ai); br = fmaf(d17.x, 0.5586467385292053f, br); bi = fmaf(d17.y, 0.5586467385292053f, bi);
      ar = fmaf(s18.x, -0.956400990486145f, ar); ai = fmaf(s18.y, -0.956400990486145f, ai); br = fmaf(d18.x, 0.29205676913261414f, br); bi = fmaf(d18.y, 0.29205676913261414f, bi);
      ar = fmaf(s19.x, 0.3758275806903839f, ar); ai = fmaf(s19.y, 0.3758275806903839f, ai); br = fmaf(d19.x, -0.926689624786377f, br); bi = fmaf(d19.y, -0.926689624786377f, bi);
      ar = fmaf(s20.x, 0.4827921986579895f, ar); ai = fmaf(s20.y, 0.4827921986579895f, ai); br = fmaf(d20.x, 0.8757349252700806f, br); bi = fmaf(d20.y, 0.8757349252700806f, bi);
      ar = fmaf(s21.x, -0.9842305779457092f, ar); ai = fmaf(s21.y, -0.9842305779457092f, ai); br = fmaf(d21.x, -0.1768902689218521f, br); bi = fmaf(d21.y, -0.1768902689218521f, bi);
      ar = fmaf(s22.x, 0.7575112581253052f, ar); ai = fmaf(s22.y, 0.7575112581253052f, ai); br = fmaf(d22.x, -0.6528221368789673f, br); bi = fmaf(d22.y, -0.6528221368789673f, bi);
      ar = fmaf(s23.x, 0.029633328318595886f, ar); ai = fmaf(s23.y, 0.029633328318595886f, ai); br = fmaf(d23.x, 0.9995608329772949f, br); bi = fmaf(d23.y, 0.9995608329772949f, bi);
      ar = fmaf(s24.x, -0.794854462146759f, ar); ai = fmaf(s24.y, -0.794854462146759f, ai); br = fmaf(d24.x, -0.6068001389503479f, br); bi = fmaf(d24.y, -0.6068001389503479f, bi);
      ar = fmaf(s25.x, 0.9720228910446167f, ar); ai = fmaf(s25.y, 0.9720228910446167f, ai); br = fmaf(d25.x, -0.2348860502243042f, br); bi = fmaf(d25.y, -0.2348860502243042f, bi);
      ar = fmaf(s26.x, -0.43006521463394165f, ar); ai = fmaf(s26.y, -0.43006521463394165f, ai); br = fmaf(d26.x, 0.9027978181838989f, br); bi = fmaf(d26.y, 0.9027978181838989f, bi);
      if (!INV) { st(19, make_float2(ar + bi, ai - br)); st(34, make_float2(ar - bi, ai + br)); }
      else { st(19, make_float2(ar - bi, ai + br)); st(34, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.7175072431564331f, ar); ai = fmaf(s1.y, -0.7175072431564331f, ai); br = fmaf(d1.x, 0.6965510249137878f, br); bi = fmaf(d1.y, 0.6965510249137878f, bi);
      ar = fmaf(s2.x, 0.029633328318595886f, ar); ai = fmaf(s2.y, 0.029633328318595886f, ai); br = fmaf(d2.x, -0.9995608329772949f, br); bi = fmaf(d2.y, -0.9995608329772949f, bi);
      ar = fmaf(s3.x, 0.674983024597168f, ar); ai = fmaf(s3.y, 0.674983024597168f, ai); br = fmaf(d3.x, 0.7378332614898682f, br); bi = fmaf(d3.y, 0.7378332614898682f, bi);
      ar = fmaf(s4.x, -0.9982437491416931f, ar); ai = fmaf(s4.y, -0.9982437491416931f, ai); br = fmaf(d4.x, -0.05924062803387642f, br); bi = fmaf(d4.y, -0.05924062803387642f, bi);
      ar = fmaf(s5.x, 0.7575112581253052f, ar); ai = fmaf(s5.y, 0.7575112581253052f, ai); br = fmaf(d5.x, -0.6528221368789673f, br); bi = fmaf(d5.y, -0.6528221368789673f, bi);
      ar = fmaf(s6.x, -0.08879589289426804f, ar); ai = fmaf(s6.y, -0.08879589289426804f, ai); br = fmaf(d6.x, 0.9960498213768005f, br); bi = fmaf(d6.y, 0.9960498213768005f, bi);
      ar = fmaf(s7.x, -0.6300878524780273f, ar); ai = fmaf(s7.y, -0.6300878524780273f, ai); br = fmaf(d7.x, -0.7765238881111145f, br); bi = fmaf(d7.y, -0.7765238881111145f, bi);
      ar = fmaf(s8.x, 0.9929810762405396f, ar); ai = fmaf(s8.y, 0.9929810762405396f, ai); br = fmaf(d8.x, 0.11827316880226135f, br); bi = fmaf(d8.y, 0.11827316880226135f, bi);
      ar = fmaf(s9.x, -0.794854462146759f, ar); ai = fmaf(s9.y, -0.794854462146759f, ai); br = fmaf(d9.x, 0.6068001389503479f, br); bi = fmaf(d9.y, 0.6068001389503479f, bi);
      ar = fmaf(s10.x, 0.14764656126499176f, ar); ai = fmaf(s10.y, 0.14764656126499176f, ai); br = fmaf(d10.x, -0.989040195941925f, br); bi = fmaf(d10.y, -0.989040195941925f, bi);
      ar = fmaf(s11.x, 0.5829795002937317f, ar); ai = fmaf(s11.y, 0.5829795002937317f, ai); br = fmaf(d11.x, 0.8124868869781494f, br); bi = fmaf(d11.y, 0.8124868869781494f, bi);
      ar = fmaf(s12.x, -0.9842305779457092f, ar); ai = fmaf(s12.y, -0.9842305779457092f, ai); br = fmaf(d12.x, -0.1768902689218521f, br); bi = fmaf(d12.y, -0.1768902689218521f, bi);
      ar = fmaf(s13.x, 0.829405665397644f, ar); ai = fmaf(s13.y, 0.829405665397644f, ai); br = fmaf(d13.x, -0.5586467385292053f, br); bi = fmaf(d13.y, -0.5586467385292053f, bi);
      ar = fmaf(s14.x, -0.2059786170721054f, ar); ai = fmaf(s14.y, -0.2059786170721054f, ai); br = fmaf(d14.x, 0.9785565137863159f, br); bi = fmaf(d14.y, 0.9785565137863159f, bi);
      ar = fmaf(s15.x, -0.5338233709335327f, ar); ai = fmaf(s15.y, -0.5338233709335327f, ai); br = fmaf(d15.x, -0.8455960154533386f, br); bi = fmaf(d15.y, -0.8455960154533386f, bi);
      ar = fmaf(s16.x, 0.9720228910446167f, ar); ai = fmaf(s16.y, 0.9720228910446167f, ai); br = fmaf(d16.x, 0.2348860502243042f, br); bi = fmaf(d16.y, 0.2348860502243042f, bi);
      ar = fmaf(s17.x, -0.8610436320304871f, ar); ai = fmaf(s17.y, -0.8610436320304871f, ai); br = fmaf(d17.x, 0.5085310935974121f, br); bi = fmaf(d17.y, 0.5085310935974121f, bi);
      ar = fmaf(s18.x, 0.26358717679977417f, ar); ai = fmaf(s18.y, 0.26358717679977417f, ai); br = fmaf(d18.x, -0.9646356105804443f, br); bi = fmaf(d18.y, -0.9646356105804443f, bi);
      ar = fmaf(s19.x, 0.4827921986579895f, ar); ai = fmaf(s19.y, 0.4827921986579895f, ai); br = fmaf(d19.x, 0.8757349252700806f, br); bi = fmaf(d19.y, 0.8757349252700806f, bi);
      ar = fmaf(s20.x, -0.956400990486145f, ar); ai = fmaf(s20.y, -0.956400990486145f, ai); br = fmaf(d20.x, -0.29205676913261414f, br); bi = fmaf(d20.y, -0.29205676913261414f, bi);
      ar = fmaf(s21.x, 0.8896570801734924f, ar); ai = fmaf(s21.y, 0.8896570801734924f, ai); br = fmaf(d21.x, -0.4566292464733124f, br); bi = fmaf(d21.y, -0.4566292464733124f, bi);
      ar = fmaf(s22.x, -0.3202698528766632f, ar); ai = fmaf(s22.y, -0.3202698528766632f, ai); br = fmaf(d22.x, 0.9473263621330261f, br); bi = fmaf(d22.y, 0.9473263621330261f, bi);
      ar = fmaf(s23.x, -0.43006521463394165f, ar); ai = fmaf(s23.y, -0.43006521463394165f, ai); br = fmaf(d23.x, -0.9027978181838989f, br); bi = fmaf(d23.y, -0.9027978181838989f, bi);
      ar = fmaf(s24.x, 0.9374196529388428f, ar); ai = fmaf(s24.y, 0.9374196529388428f, ai); br = fmaf(d24.x, 0.3482016324996948f, br); bi = fmaf(d24.y, 0.3482016324996948f, bi);
      ar = fmaf(s25.x, -0.9151456356048584f, ar); ai = fmaf(s25.y, -0.9151456356048584f, ai); br = fmaf(d25.x, 0.4031234383583069f, br); bi = fmaf(d25.y, 0.4031234383583069f, bi);
      ar = fmaf(s26.x, 0.3758275806903839f, ar); ai = fmaf(s26.y, 0.3758275806903839f, ai); br = fmaf(d26.x, -0.926689624786377f, br); bi = fmaf(d26.y, -0.926689624786377f, bi);
      if (!INV) { st(20, make_float2(ar + bi, ai - br)); st(33, make_float2(ar - bi, ai + br)); }
      else { st(20, make_float2(ar - bi, ai + br)); st(33, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.794854462146759f, ar); ai = fmaf(s1.y, -0.794854462146759f, ai); br = fmaf(d1.x, 0.6068001389503479f, br); bi = fmaf(d1.y, 0.6068001389503479f, bi);
      ar = fmaf(s2.x, 0.26358717679977417f, ar); ai = fmaf(s2.y, 0.26358717679977417f, ai); br = fmaf(d2.x, -0.9646356105804443f, br); bi = fmaf(d2.y, -0.9646356105804443f, bi);
      ar = fmaf(s3.x, 0.3758275806903839f, ar); ai = fmaf(s3.y, 0.3758275806903839f, ai); br = fmaf(d3.x, 0.926689624786377f, br); bi = fmaf(d3.y, 0.926689624786377f, bi);
      ar = fmaf(s4.x, -0.8610436320304871f, ar); ai = fmaf(s4.y, -0.8610436320304871f, ai); br = fmaf(d4.x, -0.5085310935974121f, br); bi = fmaf(d4.y, -0.5085310935974121f, bi);
      ar = fmaf(s5.x, 0.9929810762405396f, ar); ai = fmaf(s5.y, 0.9929810762405396f, ai); br = fmaf(d5.x, -0.11827316880226135f, br); bi = fmaf(d5.y, -0.11827316880226135f, bi);
      ar = fmaf(s6.x, -0.7175072431564331f, ar); ai = fmaf(s6.y, -0.7175072431564331f, ai); br = fmaf(d6.x, 0.6965510249137878f, br); bi = fmaf(d6.y, 0.6965510249137878f, bi);
      ar = fmaf(s7.x, 0.14764656126499176f, ar); ai = fmaf(s7.y, 0.14764656126499176f, ai); br = fmaf(d7.x, -0.989040195941925f, br); bi = fmaf(d7.y, -0.989040195941925f, bi);
      ar = fmaf(s8.x, 0.4827921986579895f, ar); ai = fmaf(s8.y, 0.4827921986579895f, ai); br = fmaf(d8.x, 0.8757349252700806f, br); bi = fmaf(d8.y, 0.8757349252700806f, bi);
      ar = fmaf(s9.x, -0.9151456356048584f, ar); ai = fmaf(s9.y, -0.9151456356048584f, ai); br = fmaf(d9.x, -0.4031234383583069f, br); bi = fmaf(d9.y, -0.4031234383583069f, bi);
      ar = fmaf(s10.x, 0.9720228910446167f, ar); ai = fmaf(s10.y, 0.9720228910446167f, ai); br = fmaf(d10.x, -0.2348860502243042f, br); bi = fmaf(d10.y, -0.2348860502243042f, bi);
      ar = fmaf(s11.x, -0.6300878524780273f, ar); ai = fmaf(s11.y, -0.6300878524780273f, ai); br = fmaf(d11.x, 0.7765238881111145f, br); bi = fmaf(d11.y, 0.7765238881111145f, bi);
      ar = fmaf(s12.x, 0.029633328318595886f, ar); ai = fmaf(s12.y, 0.029633328318595886f, ai); br = fmaf(d12.x, -0.9995608329772949f, br); bi = fmaf(d12.y, -0.9995608329772949f, bi);
      ar = fmaf(s13.x, 0.5829795002937317f, ar); ai = fmaf(s13.y, 0.5829795002937317f, ai); br = fmaf(d13.x, 0.8124868869781494f, br); bi = fmaf(d13.y, 0.8124868869781494f, bi);
      ar = fmaf(s14.x, -0.956400990486145f, ar); ai = fmaf(s14.y, -0.956400990486145f, ai); br = fmaf(d14.x, -0.29205676913261414f, br); bi = fmaf(d14.y, -0.29205676913261414f, bi);
      ar = fmaf(s15.x, 0.9374196529388428f, ar); ai = fmaf(s15.y, 0.9374196529388428f, ai); br = fmaf(d15.x, -0.3482016324996948f, br); bi = fmaf(d15.y, -0.3482016324996948f, bi);
      ar = fmaf(s16.x, -0.5338233709335327f, ar); ai = fmaf(s16.y, -0.5338233709335327f, ai); br = fmaf(d16.x, 0.8455960154533386f, br); bi = fmaf(d16.y, 0.8455960154533386f, bi);
      ar = fmaf(s17.x, -0.08879589289426804f, ar); ai = fmaf(s17.y, -0.08879589289426804f, ai); br = fmaf(d17.x, -0.9960498213768005f, br); bi = fmaf(d17.y, -0.9960498213768005f, bi);
      ar = fmaf(s18.x, 0.674983024597168f, ar); ai = fmaf(s18.y, 0.674983024597168f, ai); br = fmaf(d18.x, 0.7378332614898682f, br); bi = fmaf(d18.y, 0.7378332614898682f, bi);
      ar = fmaf(s19.x, -0.9842305779457092f, ar); ai = fmaf(s19.y, -0.9842305779457092f, ai); br = fmaf(d19.x, -0.1768902689218521f, br); bi = fmaf(d19.y, -0.1768902689218521f, bi);
      ar = fmaf(s20.x, 0.8896570801734924f, ar); ai = fmaf(s20.y, 0.8896570801734924f, ai); br = fmaf(d20.x, -0.4566292464733124f, br); bi = fmaf(d20.y, -0.4566292464733124f, bi);
      ar = fmaf(s21.x, -0.43006521463394165f, ar); ai = fmaf(s21.y, -0.43006521463394165f, ai); br = fmaf(d21.x, 0.9027978181838989f, br); bi = fmaf(d21.y, 0.9027978181838989f, bi);
      ar = fmaf(s22.x, -0.2059786170721054f, ar); ai = fmaf(s22.y, -0.2059786170721054f, ai); br = fmaf(d22.x, -0.9785565137863159f, br); bi = fmaf(d22.y, -0.9785565137863159f, bi);
      ar = fmaf(s23.x, 0.7575112581253052f, ar); ai = fmaf(s23.y, 0.7575112581253052f, ai); br = fmaf(d23.x, 0.6528221368789673f, br); bi = fmaf(d23.y, 0.6528221368789673f, bi);
      ar = fmaf(s24.x, -0.9982437491416931f, ar); ai = fmaf(s24.y, -0.9982437491416931f, ai); br = fmaf(d24.x, -0.05924062803387642f, br); bi = fmaf(d24.y, -0.05924062803387642f, bi);
      ar = fmaf(s25.x, 0.829405665397644f, ar); ai = fmaf(s25.y, 0.829405665397644f, ai); br = fmaf(d25.x, -0.5586467385292053f, br); bi = fmaf(d25.y, -0.5586467385292053f, bi);
      ar = fmaf(s26.x, -0.3202698528766632f, ar); ai = fmaf(s26.y, -0.3202698528766632f, ai); br = fmaf(d26.x, 0.9473263621330261f, br); bi = fmaf(d26.y, 0.9473263621330261f, bi);
      if (!INV) { st(21, make_float2(ar + bi, ai - br)); st(32, make_float2(ar - bi, ai + br)); }
      else { st(21, make_float2(ar - bi, ai + br)); st(32, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.8610436320304871f, ar); ai = fmaf(s1.y, -0.8610436320304871f, ai); br = fmaf(d1.x, 0.5085310935974121f, br); bi = fmaf(d1.y, 0.5085310935974121f, bi);
      ar = fmaf(s2.x, 0.4827921986579895f, ar); ai = fmaf(s2.y, 0.4827921986579895f, ai); br = fmaf(d2.x, -0.8757349252700806f, br); bi = fmaf(d2.y, -0.8757349252700806f, bi);
      ar = fmaf(s3.x, 0.029633328318595886f, ar); ai = fmaf(s3.y, 0.029633328318595886f, ai); br = fmaf(d3.x, 0.9995608329772949f, br); bi = fmaf(d3.y, 0.9995608329772949f, bi);
      ar = fmaf(s4.x, -0.5338233709335327f, ar); ai = fmaf(s4.y, -0.5338233709335327f, ai); br = fmaf(d4.x, -0.8455960154533386f, br); bi = fmaf(d4.y, -0.8455960154533386f, bi);
      ar = fmaf(s5.x, 0.8896570801734924f, ar); ai = fmaf(s5.y, 0.8896570801734924f, ai); br = fmaf(d5.x, 0.4566292464733124f, br); bi = fmaf(d5.y, 0.4566292464733124f, bi);
      ar = fmaf(s6.x, -0.9982437491416931f, ar); ai = fmaf(s6.y, -0.9982437491416931f, ai); br = fmaf(d6.x, 0.05924062803387642f, br); bi = fmaf(d6.y, 0.05924062803387642f, bi);
      ar = fmaf(s7.x, 0.829405665397644f, ar); ai = fmaf(s7.y, 0.829405665397644f, ai); br = fmaf(d7.x, -0.5586467385292053f, br); bi = fmaf(d7.y, -0.5586467385292053f, bi);
      ar = fmaf(s8.x, -0.43006521463394165f, ar); ai = fmaf(s8.y, -0.43006521463394165f, ai); br = fmaf(d8.x, 0.9027978181838989f, br); bi = fmaf(d8.y, 0.9027978181838989f, bi);
      ar = fmaf(s9.x, -0.08879589289426804f, ar); ai = fmaf(s9.y, -0.08879589289426804f, ai); br = fmaf(d9.x, -0.9960498213768005f, br); bi = fmaf(d9.y, -0.9960498213768005f, bi);
      ar = fmaf(s10.x, 0.5829795002937317f, ar); ai = fmaf(s10.y, 0.5829795002937317f, ai); br = fmaf(d10.x, 0.8124868869781494f, br); bi = fmaf(d10.y, 0.8124868869781494f, bi);
      ar = fmaf(s11.x, -0.9151456356048584f, ar); ai = fmaf(s11.y, -0.9151456356048584f, ai); br = fmaf(d11.x, -0.4031234383583069f, br); bi = fmaf(d11.y, -0.4031234383583069f, bi);
      ar = fmaf(s12.x, 0.9929810762405396f, ar); ai = fmaf(s12.y, 0.9929810762405396f, ai); br = fmaf(d12.x, -0.11827316880226135f, br); bi = fmaf(d12.y, -0.11827316880226135f, bi);
      ar = fmaf(s13.x, -0.794854462146759f, ar); ai = fmaf(s13.y, -0.794854462146759f, ai); br = fmaf(d13.x, 0.6068001389503479f, br); bi = fmaf(d13.y, 0.6068001389503479f, bi);
      ar = fmaf(s14.x, 0.3758275806903839f, ar); ai = fmaf(s14.y, 0.3758275806903839f, ai); br = fmaf(d14.x, -0.926689624786377f, br); bi = fmaf(d14.y, -0.926689624786377f, bi);
      ar = fmaf(s15.x, 0.14764656126499176f, ar); ai = fmaf(s15.y, 0.14764656126499176f, ai); br = fmaf(d15.x, 0.989040195941925f, br); bi = fmaf(d15.y, 0.989040195941925f, bi);
      ar = fmaf(s16.x, -0.6300878524780273f, ar); ai = fmaf(s16.y, -0.6300878524780273f, ai); br = fmaf(d16.x, -0.7765238881111145f, br); bi = fmaf(d16.y, -0.7765238881111145f, bi);
      ar = fmaf(s17.x, 0.9374196529388428f, ar); ai = fmaf(s17.y, 0.9374196529388428f, ai); br = fmaf(d17.x, 0.3482016324996948f, br); bi = fmaf(d17.y, 0.3482016324996948f, bi);
      ar = fmaf(s18.x, -0.9842305779457092f, ar); ai = fmaf(s18.y, -0.9842305779457092f, ai); br = fmaf(d18.x, 0.1768902689218521f, br); bi = fmaf(d18.y, 0.1768902689218521f, bi);
      ar = fmaf(s19.x, 0.7575112581253052f, ar); ai = fmaf(s19.y, 0.7575112581253052f, ai); br = fmaf(d19.x, -0.6528221368789673f, br); bi = fmaf(d19.y, -0.6528221368789673f, bi);
      ar = fmaf(s20.x, -0.3202698528766632f, ar); ai = fmaf(s20.y, -0.3202698528766632f, ai); br = fmaf(d20.x, 0.9473263621330261f, br); bi = fmaf(d20.y, 0.9473263621330261f, bi);
      ar = fmaf(s21.x, -0.2059786170721054f, ar); ai = fmaf(s21.y, -0.2059786170721054f, ai); br = fmaf(d21.x, -0.9785565137863159f, br); bi = fmaf(d21.y, -0.9785565137863159f, bi);
      ar = fmaf(s22.x, 0.674983024597168f, ar); ai = fmaf(s22.y, 0.674983024597168f, ai); br = fmaf(d22.x, 0.7378332614898682f, br); bi = fmaf(d22.y, 0.7378332614898682f, bi);
      ar = fmaf(s23.x, -0.956400990486145f, ar); ai = fmaf(s23.y, -0.956400990486145f, ai); br = fmaf(d23.x, -0.29205676913261414f, br); bi = fmaf(d23.y, -0.29205676913261414f, bi);
      ar = fmaf(s24.x, 0.9720228910446167f, ar); ai = fmaf(s24.y, 0.9720228910446167f, ai); br = fmaf(d24.x, -0.2348860502243042f, br); bi = fmaf(d24.y, -0.2348860502243042f, bi);
      ar = fmaf(s25.x, -0.7175072431564331f, ar); ai = fmaf(s25.y, -0.7175072431564331f, ai); br = fmaf(d25.x, 0.6965510249137878f, br); bi = fmaf(d25.y, 0.6965510249137878f, bi);
      ar = fmaf(s26.x, 0.26358717679977417f, ar); ai = fmaf(s26.y, 0.26358717679977417f, ai); br = fmaf(d26.x, -0.9646356105804443f, br); bi = fmaf(d26.y, -0.9646356105804443f, bi);
      if (!INV) { st(22, make_float2(ar + bi, ai - br)); st(31, make_float2(ar - bi, ai + br)); }
      else { st(22, make_float2(ar - bi, ai + br)); st(31, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.9151456356048584f, ar); ai = fmaf(s1.y, -0.9151456356048584f, ai); br = fmaf(d1.x, 0.4031234383583069f, br); bi = fmaf(d1.y, 0.4031234383583069f, bi);
      ar = fmaf(s2.x, 0.674983024597168f, ar); ai = fmaf(s2.y, 0.674983024597168f, ai); br = fmaf(d2.x, -0.7378332614898682f, br); bi = fmaf(d2.y, -0.7378332614898682f, bi);
      ar = fmaf(s3.x, -0.3202698528766632f, ar); ai = fmaf(s3.y, -0.3202698528766632f, ai); br = fmaf(d3.x, 0.9473263621330261f, br); bi = fmaf(d3.y, 0.9473263621330261f, bi);
      ar = fmaf(s4.x, -0.08879589289426804f, ar); ai = fmaf(s4.y, -0.08879589289426804f, ai); br = fmaf(d4.x, -0.9960498213768005f, br); bi = fmaf(d4.y, -0.9960498213768005f, bi);
      ar = fmaf(s5.x, 0.4827921986579895f, ar); ai = fmaf(s5.y, 0.4827921986579895f, ai); br = fmaf(d5.x, 0.8757349252700806f, br); bi = fmaf(d5.y, 0.8757349252700806f, bi);
      ar = fmaf(s6.x, -0.794854462146759f, ar); ai = fmaf(s6.y, -0.794854462146759f, ai); br = fmaf(d6.x, -0.6068001389503479f, br); bi = fmaf(d6.y, -0.6068001389503479f, bi);
      ar = fmaf(s7.x, 0.9720228910446167f, ar); ai = fmaf(s7.y, 0.9720228910446167f, ai); br = fmaf(d7.x, 0.2348860502243042f, br); bi = fmaf(d7.y, 0.2348860502243042f, bi);
      ar = fmaf(s8.x, -0.9842305779457092f, ar); ai = fmaf(s8.y, -0.9842305779457092f, ai); br = fmaf(d8.x, 0.1768902689218521f, br); bi = fmaf(d8.y, 0.1768902689218521f, bi);
      ar = fmaf(s9.x, 0.829405665397644f, ar); ai = fmaf(s9.y, 0.829405665397644f, ai); br = fmaf(d9.x, -0.5586467385292053f, br); bi = fmaf(d9.y, -0.5586467385292053f, bi);
      ar = fmaf(s10.x, -0.5338233709335327f, ar); ai = fmaf(s10.y, -0.5338233709335327f, ai); br = fmaf(d10.x, 0.8455960154533386f, br); bi = fmaf(d10.y, 0.8455960154533386f, bi);
      ar = fmaf(s11.x, 0.14764656126499176f, ar); ai = fmaf(s11.y, 0.14764656126499176f, ai); br = fmaf(d11.x, -0.989040195941925f, br); bi = fmaf(d11.y, -0.989040195941925f, bi);
      ar = fmaf(s12.x, 0.26358717679977417f, ar); ai = fmaf(s12.y, 0.26358717679977417f, ai); br = fmaf(d12.x, 0.9646356105804443f, br); bi = fmaf(d12.y, 0.9646356105804443f, bi);
      ar = fmaf(s13.x, -0.6300878524780273f, ar); ai = fmaf(s13.y, -0.6300878524780273f, ai); br = fmaf(d13.x, -0.7765238881111145f, br); bi = fmaf(d13.y, -0.7765238881111145f, bi);
      ar = fmaf(s14.x, 0.8896570801734924f, ar); ai = fmaf(s14.y, 0.8896570801734924f, ai); br = fmaf(d14.x, 0.4566292464733124f, br); bi = fmaf(d14.y, 0.4566292464733124f, bi);
      ar = fmaf(s15.x, -0.9982437491416931f, ar); ai = fmaf(s15.y, -0.9982437491416931f, ai); br = fmaf(d15.x, -0.05924062803387642f, br); bi = fmaf(d15.y, -0.05924062803387642f, bi);
      ar = fmaf(s16.x, 0.9374196529388428f, ar); ai = fmaf(s16.y, 0.9374196529388428f, ai); br = fmaf(d16.x, -0.3482016324996948f, br); bi = fmaf(d16.y, -0.3482016324996948f, bi);
      ar = fmaf(s17.x, -0.7175072431564331f, ar); ai = fmaf(s17.y, -0.7175072431564331f, ai); br = fmaf(d17.x, 0.6965510249137878f, br); bi = fmaf(d17.y, 0.6965510249137878f, bi);
      ar = fmaf(s18.x, 0.3758275806903839f, ar); ai = fmaf(s18.y, 0.3758275806903839f, ai); br = fmaf(d18.x, -0.926689624786377f, br); bi = fmaf(d18.y, -0.926689624786377f, bi);
      ar = fmaf(s19.x, 0.029633328318595886f, ar); ai = fmaf(s19.y, 0.029633328318595886f, ai); br = fmaf(d19.x, 0.9995608329772949f, br); bi = fmaf(d19.y, 0.9995608329772949f, bi);
      ar = fmaf(s20.x, -0.43006521463394165f, ar); ai = fmaf(s20.y, -0.43006521463394165f, ai); br = fmaf(d20.x, -0.9027978181838989f, br); bi = fmaf(d20.y, -0.9027978181838989f, bi);
      ar = fmaf(s21.x, 0.7575112581253052f, ar); ai = fmaf(s21.y, 0.7575112581253052f, ai); br = fmaf(d21.x, 0.6528221368789673f, br); bi = fmaf(d21.y, 0.6528221368789673f, bi);
      ar = fmaf(s22.x, -0.956400990486145f, ar); ai = fmaf(s22.y, -0.956400990486145f, ai); br = fmaf(d22.x, -0.29205676913261414f, br); bi = fmaf(d22.y, -0.29205676913261414f, bi);
      ar = fmaf(s23.x, 0.9929810762405396f, ar); ai = fmaf(s23.y, 0.9929810762405396f, ai); br = fmaf(d23.x, -0.11827316880226135f, br); bi = fmaf(d23.y, -0.11827316880226135f, bi);
      ar = fmaf(s24.x, -0.8610436320304871f, ar); ai = fmaf(s24.y, -0.8610436320304871f, ai); br = fmaf(d24.x, 0.5085310935974121f, br); bi = fmaf(d24.y, 0.5085310935974121f, bi);
      ar = fmaf(s25.x, 0.5829795002937317f, ar); ai = fmaf(s25.y, 0.5829795002937317f, ai); br = fmaf(d25.x, -0.8124868869781494f, br); bi = fmaf(d25.y, -0.8124868869781494f, bi);
      ar = fmaf(s26.x, -0.2059786170721054f, ar); ai = fmaf(s26.y, -0.2059786170721054f, ai); br = fmaf(d26.x, 0.9785565137863159f, br); bi = fmaf(d26.y, 0.9785565137863159f, bi);
      if (!INV) { st(23, make_float2(ar + bi, ai - br)); st(30, make_float2(ar - bi, ai + br)); }
      else { st(23, make_float2(ar - bi, ai + br)); st(30, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.956400990486145f, ar); ai = fmaf(s1.y, -0.956400990486145f, ai); br = fmaf(d1.x, 0.29205676913261414f, br); bi = fmaf(d1.y, 0.29205676913261414f, bi);
      ar = fmaf(s2.x, 0.829405665397644f, ar); ai = fmaf(s2.y, 0.829405665397644f, ai); br = fmaf(d2.x, -0.5586467385292053f, br); bi = fmaf(d2.y, -0.5586467385292053f, bi);
      ar = fmaf(s3.x, -0.6300878524780273f, ar); ai = fmaf(s3.y, -0.6300878524780273f, ai); br = fmaf(d3.x, 0.7765238881111145f, br); bi = fmaf(d3.y, 0.7765238881111145f, bi);
      ar = fmaf(s4.x, 0.3758275806903839f, ar); ai = fmaf(s4.y, 0.3758275806903839f, ai); br = fmaf(d4.x, -0.926689624786377f, br); bi = fmaf(d4.y, -0.926689624786377f, bi);
      ar = fmaf(s5.x, -0.08879589289426804f, ar); ai = fmaf(s5.y, -0.08879589289426804f, ai); br = fmaf(d5.x, 0.9960498213768005f, br); bi = fmaf(d5.y, 0.9960498213768005f, bi);
      ar = fmaf(s6.x, -0.2059786170721054f, ar); ai = fmaf(s6.y, -0.2059786170721054f, ai); br = fmaf(d6.x, -0.9785565137863159f, br); bi = fmaf(d6.y, -0.9785565137863159f, bi);
      ar = fmaf(s7.x, 0.4827921986579895f, ar); ai = fmaf(s7.y, 0.4827921986579895f, ai); br = fmaf(d7.x, 0.8757349252700806f, br); bi = fmaf(d7.y, 0.8757349252700806f, bi);
      ar = fmaf(s8.x, -0.7175072431564331f, ar); ai = fmaf(s8.y, -0.7175072431564331f, ai); br = fmaf(d8.x, -0.6965510249137878f, br); bi = fmaf(d8.y, -0.6965510249137878f, bi);
      ar = fmaf(s9.x, 0.8896570801734924f, ar); ai = fmaf(s9.y, 0.8896570801734924f, ai); br = fmaf(d9.x, 0.4566292464733124f, br); bi = fmaf(d9.y, 0.4566292464733124f, bi);
      ar = fmaf(s10.x, -0.9842305779457092f, ar); ai = fmaf(s10.y, -0.9842305779457092f, ai); br = fmaf(d10.x, -0.1768902689218521f, br); bi = fmaf(d10.y, -0.1768902689218521f, bi);
      ar = fmaf(s11.x, 0.9929810762405396f, ar); ai = fmaf(s11.y, 0.9929810762405396f, ai); br = fmaf(d11.x, -0.11827316880226135f, br); bi = fmaf(d11.y, -0.11827316880226135f, bi);
      ar = fmaf(s12.x, -0.9151456356048584f, ar); ai = fmaf(s12.y, -0.9151456356048584f, ai); br = fmaf(d12.x, 0.4031234383583069f, br); bi = fmaf(d12.y, 0.4031234383583069f, bi);
      ar = fmaf(s13.x, 0.7575112581253052f, ar); ai = fmaf(s13.y, 0.7575112581253052f, ai); br = fmaf(d13.x, -0.6528221368789673f, br); bi = fmaf(d13.y, -0.6528221368789673f, bi);
      ar = fmaf(s14.x, -0.5338233709335327f, ar); ai = fmaf(s14.y, -0.5338233709335327f, ai); br = fmaf(d14.x, 0.8455960154533386f, br); bi = fmaf(d14.y, 0.8455960154533386f, bi);
      ar = fmaf(s15.x, 0.26358717679977417f, ar); ai = fmaf(s15.y, 0.26358717679977417f, ai); br = fmaf(d15.x, -0.9646356105804443f, br); bi = fmaf(d15.y, -0.9646356105804443f, bi);
      ar = fmaf(s16.x, 0.029633328318595886f, ar); ai = fmaf(s16.y, 0.029633328318595886f, ai); br = fmaf(d16.x, 0.9995608329772949f, br); bi = fmaf(d16.y, 0.9995608329772949f, bi);
      ar = fmaf(s17.x, -0.3202698528766632f, ar); ai = fmaf(s17.y, -0.3202698528766632f, ai); br = fmaf(d17.x, -0.9473263621330261f, br); bi = fmaf(d17.y, -0.9473263621330261f, bi);
      ar = fmaf(s18.x, 0.5829795002937317f, ar); ai = fmaf(s18.y, 0.5829795002937317f, ai); br = fmaf(d18.x, 0.8124868869781494f, br); bi = fmaf(d18.y, 0.8124868869781494f, bi);
      ar = fmaf(s19.x, -0.794854462146759f, ar); ai = fmaf(s19.y, -0.794854462146759f, ai); br = fmaf(d19.x, -0.6068001389503479f, br); bi = fmaf(d19.y, -0.6068001389503479f, bi);
      ar = fmaf(s20.x, 0.9374196529388428f, ar); ai = fmaf(s20.y, 0.9374196529388428f, ai); br = fmaf(d20.x, 0.3482016324996948f, br); bi = fmaf(d20.y, 0.3482016324996948f, bi);
      ar = fmaf(s21.x, -0.9982437491416931f, ar); ai = fmaf(s21.y, -0.9982437491416931f, ai); br = fmaf(d21.x, -0.05924062803387642f, br); bi = fmaf(d21.y, -0.05924062803387642f, bi);
      ar = fmaf(s22.x, 0.9720228910446167f, ar); ai = fmaf(s22.y, 0.9720228910446167f, ai); br = fmaf(d22.x, -0.2348860502243042f, br); bi = fmaf(d22.y, -0.2348860502243042f, bi);
      ar = fmaf(s23.x, -0.8610436320304871f, ar); ai = fmaf(s23.y, -0.8610436320304871f, ai); br = fmaf(d23.x, 0.5085310935974121f, br); bi = fmaf(d23.y, 0.5085310935974121f, bi);
      ar = fmaf(s24.x, 0.674983024597168f, ar); ai = fmaf(s24.y, 0.674983024597168f, ai); br = fmaf(d24.x, -0.7378332614898682f, br); bi = fmaf(d24.y, -0.7378332614898682f, bi);
      ar = fmaf(s25.x, -0.43006521463394165f, ar); ai = fmaf(s25.y, -0.43006521463394165f, ai); br = fmaf(d25.x, 0.9027978181838989f, br); bi = fmaf(d25.y, 0.9027978181838989f, bi);
      ar = fmaf(s26.x, 0.14764656126499176f, ar); ai = fmaf(s26.y, 0.14764656126499176f, ai); br = fmaf(d26.x, -0.989040195941925f, br); bi = fmaf(d26.y, -0.989040195941925f, bi);
      if (!INV) { st(24, make_float2(ar + bi, ai - br)); st(29, make_float2(ar - bi, ai + br)); }
      else { st(24, make_float2(ar - bi, ai + br)); st(29, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.9842305779457092f, ar); ai = fmaf(s1.y, -0.9842305779457092f, ai); br = fmaf(d1.x, 0.1768902689218521f, br); bi = fmaf(d1.y, 0.1768902689218521f, bi);
      ar = fmaf(s2.x, 0.9374196529388428f, ar); ai = fmaf(s2.y, 0.9374196529388428f, ai); br = fmaf(d2.x, -0.3482016324996948f, br); bi = fmaf(d2.y, -0.3482016324996948f, bi);
      ar = fmaf(s3.x, -0.8610436320304871f, ar); ai = fmaf(s3.y, -0.8610436320304871f, ai); br = fmaf(d3.x, 0.5085310935974121f, br); bi = fmaf(d3.y, 0.5085310935974121f, bi);
      ar = fmaf(s4.x, 0.7575112581253052f, ar); ai = fmaf(s4.y, 0.7575112581253052f, ai); br = fmaf(d4.x, -0.6528221368789673f, br); bi = fmaf(d4.y, -0.6528221368789673f, bi);
      ar = fmaf(s5.x, -0.6300878524780273f, ar); ai = fmaf(s5.y, -0.6300878524780273f, ai); br = fmaf(d5.x, 0.7765238881111145f, br); bi = fmaf(d5.y, 0.7765238881111145f, bi);
      ar = fmaf(s6.x, 0.4827921986579895f, ar); ai = fmaf(s6.y, 0.4827921986579895f, ai); br = fmaf(d6.x, -0.8757349252700806f, br); bi = fmaf(d6.y, -0.8757349252700806f, bi);
      ar = fmaf(s7.x, -0.3202698528766632f, ar); ai = fmaf(s7.y, -0.3202698528766632f, ai); br = fmaf(d7.x, 0.9473263621330261f, br); bi = fmaf(d7.y, 0.9473263621330261f, bi);
      ar = fmaf(s8.x, 0.14764656126499176f, ar); ai = fmaf(s8.y, 0.14764656126499176f, ai); br = fmaf(d8.x, -0.989040195941925f, br); bi = fmaf(d8.y, -0.989040195941925f, bi);
      ar = fmaf(s9.x, 0.029633328318595886f, ar); ai = fmaf(s9.y, 0.029633328318595886f, ai); br = fmaf(d9.x, 0.9995608329772949f, br); bi = fmaf(d9.y, 0.9995608329772949f, bi);
      ar = fmaf(s10.x, -0.2059786170721054f, ar); ai = fmaf(s10.y, -0.2059786170721054f, ai); br = fmaf(d10.x, -0.9785565137863159f, br); bi = fmaf(d10.y, -0.9785565137863159f, bi);
      ar = fmaf(s11.x, 0.3758275806903839f, ar); ai = fmaf(s11.y, 0.3758275806903839f, ai); br = fmaf(d11.x, 0.926689624786377f, br); bi = fmaf(d11.y, 0.926689624786377f, bi);
      ar = fmaf(s12.x, -0.5338233709335327f, ar); ai = fmaf(s12.y, -0.5338233709335327f, ai); br = fmaf(d12.x, -0.8455960154533386f, br); bi = fmaf(d12.y, -0.8455960154533386f, bi);
      ar = fmaf(s13.x, 0.674983024597168f, ar); ai = fmaf(s13.y, 0.674983024597168f, ai); br = fmaf(d13.x, 0.7378332614898682f, br); bi = fmaf(d13.y, 0.7378332614898682f, bi);
      ar = fmaf(s14.x, -0.794854462146759f, ar); ai = fmaf(s14.y, -0.794854462146759f, ai); br = fmaf(d14.x, -0.6068001389503479f, br); bi = fmaf(d14.y, -0.6068001389503479f, bi);
      ar = fmaf(s15.x, 0.8896570801734924f, ar); ai = fmaf(s15.y, 0.8896570801734924f, ai); br = fmaf(d15.x, 0.4566292464733124f, br); bi = fmaf(d15.y, 0.4566292464733124f, bi);
      ar = fmaf(s16.x, -0.956400990486145f, ar); ai = fmaf(s16.y, -0.956400990486145f, ai); br = fmaf(d16.x, -0.29205676913261414f, br); bi = fmaf(d16.y, -0.29205676913261414f, bi);
      ar = fmaf(s17.x, 0.9929810762405396f, ar); ai = fmaf(s17.y, 0.9929810762405396f, ai); br = fmaf(d17.x, 0.11827316880226135f, br); bi = fmaf(d17.y, 0.11827316880226135f, bi);
      ar = fmaf(s18.x, -0.9982437491416931f, ar); ai = fmaf(s18.y, -0.9982437491416931f, ai); br = fmaf(d18.x, 0.05924062803387642f, br); bi = fmaf(d18.y, 0.05924062803387642f, bi);
      ar = fmaf(s19.x, 0.9720228910446167f, ar); ai = fmaf(s19.y, 0.9720228910446167f, ai); br = fmaf(d19.x, -0.2348860502243042f, br); bi = fmaf(d19.y, -0.2348860502243042f, bi);
      ar = fmaf(s20.x, -0.9151456356048584f, ar); ai = fmaf(s20.y, -0.9151456356048584f, ai); br = fmaf(d20.x, 0.4031234383583069f, br); bi = fmaf(d20.y, 0.4031234383583069f, bi);
      ar = fmaf(s21.x, 0.829405665397644f, ar); ai = fmaf(s21.y, 0.829405665397644f, ai); br = fmaf(d21.x, -0.5586467385292053f, br); bi = fmaf(d21.y, -0.5586467385292053f, bi);
      ar = fmaf(s22.x, -0.7175072431564331f, ar); ai = fmaf(s22.y, -0.7175072431564331f, ai); br = fmaf(d22.x, 0.6965510249137878f, br); bi = fmaf(d22.y, 0.6965510249137878f, bi);
      ar = fmaf(s23.x, 0.5829795002937317f, ar); ai = fmaf(s23.y, 0.5829795002937317f, ai); br = fmaf(d23.x, -0.8124868869781494f, br); bi = fmaf(d23.y, -0.8124868869781494f, bi);
      ar = fmaf(s24.x, -0.43006521463394165f, ar); ai = fmaf(s24.y, -0.43006521463394165f, ai); br = fmaf(d24.x, 0.9027978181838989f, br); bi = fmaf(d24.y, 0.9027978181838989f, bi);
      ar = fmaf(s25.x, 0.26358717679977417f, ar); ai = fmaf(s25.y, 0.26358717679977417f, ai); br = fmaf(d25.x, -0.9646356105804443f, br); bi = fmaf(d25.y, -0.9646356105804443f, bi);
      ar = fmaf(s26.x, -0.08879589289426804f, ar); ai = fmaf(s26.y, -0.08879589289426804f, ai); br = fmaf(d26.x, 0.9960498213768005f, br); bi = fmaf(d26.y, 0.9960498213768005f, bi);
      if (!INV) { st(25, make_float2(ar + bi, ai - br)); st(28, make_float2(ar - bi, ai + br)); }
      else { st(25, make_float2(ar - bi, ai + br)); st(28, make_float2(ar + bi, ai - br)); }
    }
    {
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      ar = fmaf(s1.x, -0.9982437491416931f, ar); ai = fmaf(s1.y, -0.9982437491416931f, ai); br = fmaf(d1.x, 0.05924062803387642f, br); bi = fmaf(d1.y, 0.05924062803387642f, bi);
      ar = fmaf(s2.x, 0.9929810762405396f, ar); ai = fmaf(s2.y, 0.9929810762405396f, ai); br = fmaf(d2.x, -0.11827316880226135f, br); bi = fmaf(d2.y, -0.11827316880226135f, bi);
      ar = fmaf(s3.x, -0.9842305779457092f, ar); ai = fmaf(s3.y, -0.9842305779457092f, ai); br = fmaf(d3.x, 0.1768902689218521f, br); bi = fmaf(d3.y, 0.1768902689218521f, bi);
      ar = fmaf(s4.x, 0.9720228910446167f, ar); ai = fmaf(s4.y, 0.9720228910446167f, ai); br = fmaf(d4.x, -0.2348860502243042f, br); bi = fmaf(d4.y, -0.2348860502243042f, bi);
      ar = fmaf(s5.x, -0.956400990486145f, ar); ai = fmaf(s5.y, -0.956400990486145f, ai); br = fmaf(d5.x, 0.29205676913261414f, br); bi = fmaf(d5.y, 0.29205676913261414f, bi);
      ar = fmaf(s6.x, 0.9374196529388428f, ar); ai = fmaf(s6.y, 0.9374196529388428f, ai); br = fmaf(d6.x, -0.3482016324996948f, br); bi = fmaf(d6.y, -0.3482016324996948f, bi);
      ar = fmaf(s7.x, -0.9151456356048584f, ar); ai = fmaf(s7.y, -0.9151456356048584f, ai); br = fmaf(d7.x, 0.4031234383583069f, br); bi = fmaf(d7.y, 0.4031234383583069f, bi);
      ar = fmaf(s8.x, 0.8896570801734924f, ar); ai = fmaf(s8.y, 0.8896570801734924f, ai); br = fmaf(d8.x, -0.4566292464733124f, br); bi = fmaf(d8.y, -0.4566292464733124f, bi);
      ar = fmaf(s9.x, -0.8610436320304871f, ar); ai = fmaf(s9.y, -0.8610436320304871f, ai); br = fmaf(d9.x, 0.5085310935974121f, br); bi = fmaf(d9.y, 0.5085310935974121f, bi);
      ar = fmaf(s10.x, 0.829405665397644f, ar); ai = fmaf(s10.y, 0.829405665397644f, ai); br = fmaf(d10.x, -0.5586467385292053f, br); bi = fmaf(d10.y, -0.5586467385292053f, bi);
      ar = fmaf(s11.x, -0.794854462146759f, ar); ai = fmaf(s11.y, -0.794854462146759f, ai); br = fmaf(d11.x, 0.6068001389503479f, br); bi = fmaf(d11.y, 0.6068001389503479f, bi);
      ar = fmaf(s12.x, 0.7575112581253052f, ar); ai = fmaf(s12.y, 0.7575112581253052f, ai); br = fmaf(d12.x, -0.6528221368789673f, br); bi = fmaf(d12.y, -0.6528221368789673f, bi);
      ar = fmaf(s13.x, -0.7175072431564331f, ar); ai = fmaf(s13.y, -0.7175072431564331f, ai); br = fmaf(d13.x, 0.6965510249137878f, br); bi = fmaf(d13.y, 0.6965510249137878f, bi);
      ar = fmaf(s14.x, 0.674983024597168f, ar); ai = fmaf(s14.y, 0.674983024597168f, ai); br = fmaf(d14.x, -0.7378332614898682f, br); bi = fmaf(d14.y, -0.7378332614898682f, bi);
      ar = fmaf(s15.x, -0.6300878524780273f, ar); ai = fmaf(s15.y, -0.6300878524780273f, ai); br = fmaf(d15.x, 0.7765238881111145f, br); bi = fmaf(d15.y, 0.7765238881111145f, bi);
      ar = fmaf(s16.x, 0.5829795002937317f, ar); ai = fmaf(s16.y, 0.5829795002937317f, ai); br = fmaf(d16.x, -0.8124868869781494f, br); bi = fmaf(d16.y, -0.8124868869781494f, bi);
      ar = fmaf(s17.x, -0.5338233709335327f, ar); ai = fmaf(s17.y, -0.5338233709335327f, ai); br = fmaf(d17.x, 0.8455960154533386f, br); bi = fmaf(d17.y, 0.8455960154533386f, bi);
      ar = fmaf(s18.x, 0.4827921986579895f, ar); ai = fmaf(s18.y, 0.4827921986579895f, ai); br = fmaf(d18.x, -0.8757349252700806f, br); bi = fmaf(d18.y, -0.8757349252700806f, bi);
      ar = fmaf(s19.x, -0.43006521463394165f, ar); ai = fmaf(s19.y, -0.43006521463394165f, ai); br = fmaf(d19.x, 0.9027978181838989f, br); bi = fmaf(d19.y, 0.9027978181838989f, bi);
      ar = fmaf(s20.x, 0.3758275806903839f, ar); ai = fmaf(s20.y, 0.3758275806903839f, ai); br = fmaf(d20.x, -0.926689624786377f, br); bi = fmaf(d20.y, -0.926689624786377f, bi);
      ar = fmaf(s21.x, -0.3202698528766632f, ar); ai = fmaf(s21.y, -0.3202698528766632f, ai); br = fmaf(d21.x, 0.9473263621330261f, br); bi = fmaf(d21.y, 0.9473263621330261f, bi);
      ar = fmaf(s22.x, 0.26358717679977417f, ar); ai = fmaf(s22.y, 0.26358717679977417f, ai); br = fmaf(d22.x, -0.9646356105804443f, br); bi = fmaf(d22.y, -0.9646356105804443f, bi);
      ar = fmaf(s23.x, -0.2059786170721054f, ar); ai = fmaf(s23.y, -0.2059786170721054f, ai); br = fmaf(d23.x, 0.9785565137863159f, br); bi = fmaf(d23.y, 0.9785565137863159f, bi);
      ar = fmaf(s24.x, 0.14764656126499176f, ar); ai = fmaf(s24.y, 0.14764656126499176f, ai); br = fmaf(d24.x, -0.989040195941925f, br); bi = fmaf(d24.y, -0.989040195941925f, bi);
      ar = fmaf(s25.x, -0.08879589289426804f, ar); ai = fmaf(s25.y, -0.08879589289426804f, ai); br = fmaf(d25.x, 0.9960498213768005f, br); bi = fmaf(d25.y, 0.9960498213768005f, bi);
      ar = fmaf(s26.x, 0.029633328318595886f, ar); ai = fmaf(s26.y, 0.029633328318595886f, ai); br = fmaf(d26.x, -0.9995608329772949f, br); bi = fmaf(d26.y, -0.9995608329772949f, bi);
      if (!INV) { st(26, make_float2(ar + bi, ai - br)); st(27, make_float2(ar - bi, ai + br)); }
      else { st(26, make_float2(ar - bi, ai + br)); st(27, make_float2(ar + bi, ai - br)); }
    }
    break;
  }
  default: break;
  }
}
__constant__ float2 c_tw53[27][27] = {{{1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 0.0f}},
  {{1.0f, 0.0f}, {0.9929810762405396f, 0.11827316880226135f}, {0.9720228910446167f, 0.2348860502243042f}, {0.9374196529388428f, 0.3482016324996948f}, {0.8896570801734924f, 0.4566292464733124f}, {0.829405665397644f, 0.5586467385292053f}, {0.7575112581253052f, 0.6528221368789673f}, {0.674983024597168f, 0.7378332614898682f}, {0.5829795002937317f, 0.8124868869781494f}, {0.4827921986579895f, 0.8757349252700806f}, {0.3758275806903839f, 0.926689624786377f}, {0.26358717679977417f, 0.9646356105804443f}, {0.14764656126499176f, 0.989040195941925f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.9151456356048584f, 0.4031234383583069f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.9842305779457092f, 0.1768902689218521f}, {-0.9982437491416931f, 0.05924062803387642f}},
  {{1.0f, 0.0f}, {0.9720228910446167f, 0.2348860502243042f}, {0.8896570801734924f, 0.4566292464733124f}, {0.7575112581253052f, 0.6528221368789673f}, {0.5829795002937317f, 0.8124868869781494f}, {0.3758275806903839f, 0.926689624786377f}, {0.14764656126499176f, 0.989040195941925f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.9982437491416931f, 0.05924062803387642f}, {-0.9842305779457092f, -0.1768902689218521f}, {-0.9151456356048584f, -0.4031234383583069f}, {-0.794854462146759f, -0.6068001389503479f}, {-0.6300878524780273f, -0.7765238881111145f}, {-0.43006521463394165f, -0.9027978181838989f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.029633328318595886f, -0.9995608329772949f}, {0.26358717679977417f, -0.9646356105804443f}, {0.4827921986579895f, -0.8757349252700806f}, {0.674983024597168f, -0.7378332614898682f}, {0.829405665397644f, -0.5586467385292053f}, {0.9374196529388428f, -0.3482016324996948f}, {0.9929810762405396f, -0.11827316880226135f}},
  {{1.0f, 0.0f}, {0.9374196529388428f, 0.3482016324996948f}, {0.7575112581253052f, 0.6528221368789673f}, {0.4827921986579895f, 0.8757349252700806f}, {0.14764656126499176f, 0.989040195941925f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.9982437491416931f, -0.05924062803387642f}, {-0.9151456356048584f, -0.4031234383583069f}, {-0.7175072431564331f, -0.6965510249137878f}, {-0.43006521463394165f, -0.9027978181838989f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.26358717679977417f, -0.9646356105804443f}, {0.5829795002937317f, -0.8124868869781494f}, {0.829405665397644f, -0.5586467385292053f}, {0.9720228910446167f, -0.2348860502243042f}, {0.9929810762405396f, 0.11827316880226135f}, {0.8896570801734924f, 0.4566292464733124f}, {0.674983024597168f, 0.7378332614898682f}, {0.3758275806903839f, 0.926689624786377f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.9842305779457092f, 0.1768902689218521f}},
  {{1.0f, 0.0f}, {0.8896570801734924f, 0.4566292464733124f}, {0.5829795002937317f, 0.8124868869781494f}, {0.14764656126499176f, 0.989040195941925f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.9842305779457092f, -0.1768902689218521f}, {-0.794854462146759f, -0.6068001389503479f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.029633328318595886f, -0.9995608329772949f}, {0.4827921986579895f, -0.8757349252700806f}, {0.829405665397644f, -0.5586467385292053f}, {0.9929810762405396f, -0.11827316880226135f}, {0.9374196529388428f, 0.3482016324996948f}, {0.674983024597168f, 0.7378332614898682f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.9151456356048584f, 0.4031234383583069f}, {-0.9982437491416931f, -0.05924062803387642f}, {-0.8610436320304871f, -0.5085310935974121f}, {-0.5338233709335327f, -0.8455960154533386f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.3758275806903839f, -0.926689624786377f}, {0.7575112581253052f, -0.6528221368789673f}, {0.9720228910446167f, -0.2348860502243042f}},
  {{1.0f, 0.0f}, {0.829405665397644f, 0.5586467385292053f}, {0.3758275806903839f, 0.926689624786377f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.9842305779457092f, 0.1768902689218521f}, {-0.9151456356048584f, -0.4031234383583069f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.029633328318595886f, -0.9995608329772949f}, {0.5829795002937317f, -0.8124868869781494f}, {0.9374196529388428f, -0.3482016324996948f}, {0.9720228910446167f, 0.2348860502243042f}, {0.674983024597168f, 0.7378332614898682f}, {0.14764656126499176f, 0.989040195941925f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.9982437491416931f, -0.05924062803387642f}, {-0.794854462146759f, -0.6068001389503479f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.26358717679977417f, -0.9646356105804443f}, {0.7575112581253052f, -0.6528221368789673f}, {0.9929810762405396f, -0.11827316880226135f}, {0.8896570801734924f, 0.4566292464733124f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.956400990486145f, 0.29205676913261414f}},
  {{1.0f, 0.0f}, {0.7575112581253052f, 0.6528221368789673f}, {0.14764656126499176f, 0.989040195941925f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.9151456356048584f, -0.4031234383583069f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.26358717679977417f, -0.9646356105804443f}, {0.829405665397644f, -0.5586467385292053f}, {0.9929810762405396f, 0.11827316880226135f}, {0.674983024597168f, 0.7378332614898682f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.9842305779457092f, 0.1768902689218521f}, {-0.8610436320304871f, -0.5085310935974121f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.3758275806903839f, -0.926689624786377f}, {0.8896570801734924f, -0.4566292464733124f}, {0.9720228910446167f, 0.2348860502243042f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.9982437491416931f, 0.05924062803387642f}, {-0.794854462146759f, -0.6068001389503479f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.4827921986579895f, -0.8757349252700806f}, {0.9374196529388428f, -0.3482016324996948f}},
  {{1.0f, 0.0f}, {0.674983024597168f, 0.7378332614898682f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.9842305779457092f, -0.1768902689218521f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.26358717679977417f, -0.9646356105804443f}, {0.8896570801734924f, -0.4566292464733124f}, {0.9374196529388428f, 0.3482016324996948f}, {0.3758275806903839f, 0.926689624786377f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.8610436320304871f, -0.5085310935974121f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.5829795002937317f, -0.8124868869781494f}, {0.9929810762405396f, -0.11827316880226135f}, {0.7575112581253052f, 0.6528221368789673f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.9982437491416931f, -0.05924062803387642f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.14764656126499176f, -0.989040195941925f}, {0.829405665397644f, -0.5586467385292053f}, {0.9720228910446167f, 0.2348860502243042f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.9151456356048584f, 0.4031234383583069f}},
  {{1.0f, 0.0f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.794854462146759f, -0.6068001389503479f}, {0.029633328318595886f, -0.9995608329772949f}, {0.829405665397644f, -0.5586467385292053f}, {0.9374196529388428f, 0.3482016324996948f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.9982437491416931f, -0.05924062803387642f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.3758275806903839f, -0.926689624786377f}, {0.9720228910446167f, -0.2348860502243042f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.9151456356048584f, -0.4031234383583069f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.674983024597168f, -0.7378332614898682f}, {0.9929810762405396f, 0.11827316880226135f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.9842305779457092f, 0.1768902689218521f}, {-0.7175072431564331f, -0.6965510249137878f}, {0.14764656126499176f, -0.989040195941925f}, {0.8896570801734924f, -0.4566292464733124f}},
  {{1.0f, 0.0f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.9982437491416931f, -0.05924062803387642f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.5829795002937317f, -0.8124868869781494f}, {0.9929810762405396f, 0.11827316880226135f}, {0.3758275806903839f, 0.926689624786377f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.9842305779457092f, -0.1768902689218521f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.674983024597168f, -0.7378332614898682f}, {0.9720228910446167f, 0.2348860502243042f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.956400990486145f, -0.29205676913261414f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.7575112581253052f, -0.6528221368789673f}, {0.9374196529388428f, 0.3482016324996948f}, {0.14764656126499176f, 0.989040195941925f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.9151456356048584f, -0.4031234383583069f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.829405665397644f, -0.5586467385292053f}, {0.8896570801734924f, 0.4566292464733124f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.8610436320304871f, 0.5085310935974121f}},
  {{1.0f, 0.0f}, {0.3758275806903839f, 0.926689624786377f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.9151456356048584f, -0.4031234383583069f}, {0.029633328318595886f, -0.9995608329772949f}, {0.9374196529388428f, -0.3482016324996948f}, {0.674983024597168f, 0.7378332614898682f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.9982437491416931f, -0.05924062803387642f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.7575112581253052f, -0.6528221368789673f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.4827921986579895f, -0.8757349252700806f}, {0.9929810762405396f, 0.11827316880226135f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.8610436320304871f, -0.5085310935974121f}, {0.14764656126499176f, -0.989040195941925f}, {0.9720228910446167f, -0.2348860502243042f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.9842305779457092f, -0.1768902689218521f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.829405665397644f, -0.5586467385292053f}},
  {{1.0f, 0.0f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.7175072431564331f, -0.6965510249137878f}, {0.4827921986579895f, -0.8757349252700806f}, {0.9720228910446167f, 0.2348860502243042f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.674983024597168f, -0.7378332614898682f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.9982437491416931f, 0.05924062803387642f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.829405665397644f, -0.5586467385292053f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.9842305779457092f, -0.1768902689218521f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.9374196529388428f, -0.3482016324996948f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.9151456356048584f, -0.4031234383583069f}, {0.14764656126499176f, -0.989040195941925f}, {0.9929810762405396f, -0.11827316880226135f}, {0.3758275806903839f, 0.926689624786377f}, {-0.794854462146759f, 0.6068001389503479f}},
  {{1.0f, 0.0f}, {0.14764656126499176f, 0.989040195941925f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.829405665397644f, -0.5586467385292053f}, {0.674983024597168f, 0.7378332614898682f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.8610436320304871f, -0.5085310935974121f}, {0.3758275806903839f, -0.926689624786377f}, {0.9720228910446167f, 0.2348860502243042f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.9982437491416931f, 0.05924062803387642f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.9374196529388428f, -0.3482016324996948f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.7175072431564331f, -0.6965510249137878f}, {0.5829795002937317f, -0.8124868869781494f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.029633328318595886f, -0.9995608329772949f}, {0.9929810762405396f, -0.11827316880226135f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.9151456356048584f, 0.4031234383583069f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.7575112581253052f, -0.6528221368789673f}},
  {{1.0f, 0.0f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.9982437491416931f, 0.05924062803387642f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.9929810762405396f, -0.11827316880226135f}, {0.14764656126499176f, 0.989040195941925f}, {-0.9842305779457092f, 0.1768902689218521f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.9720228910446167f, -0.2348860502243042f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.956400990486145f, 0.29205676913261414f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.9374196529388428f, -0.3482016324996948f}, {0.3758275806903839f, 0.926689624786377f}, {-0.9151456356048584f, 0.4031234383583069f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.8896570801734924f, -0.4566292464733124f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.829405665397644f, -0.5586467385292053f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.7575112581253052f, -0.6528221368789673f}, {0.674983024597168f, 0.7378332614898682f}, {-0.7175072431564331f, 0.6965510249137878f}},
  {{1.0f, 0.0f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.26358717679977417f, -0.9646356105804443f}, {0.9374196529388428f, 0.3482016324996948f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.8610436320304871f, -0.5085310935974121f}, {0.5829795002937317f, -0.8124868869781494f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.829405665397644f, -0.5586467385292053f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.9151456356048584f, 0.4031234383583069f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.9720228910446167f, -0.2348860502243042f}, {0.14764656126499176f, 0.989040195941925f}, {-0.9982437491416931f, 0.05924062803387642f}, {0.029633328318595886f, -0.9995608329772949f}, {0.9929810762405396f, 0.11827316880226135f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.956400990486145f, -0.29205676913261414f}, {0.3758275806903839f, -0.926689624786377f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.794854462146759f, -0.6068001389503479f}, {0.674983024597168f, -0.7378332614898682f}},
  {{1.0f, 0.0f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.9151456356048584f, -0.4031234383583069f}, {0.5829795002937317f, -0.8124868869781494f}, {0.674983024597168f, 0.7378332614898682f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.9929810762405396f, -0.11827316880226135f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.956400990486145f, -0.29205676913261414f}, {0.4827921986579895f, -0.8757349252700806f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.9720228910446167f, -0.2348860502243042f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.3758275806903839f, -0.926689624786377f}, {0.829405665397644f, 0.5586467385292053f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.9374196529388428f, -0.3482016324996948f}, {0.14764656126499176f, 0.989040195941925f}, {-0.9982437491416931f, -0.05924062803387642f}, {0.26358717679977417f, -0.9646356105804443f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.6300878524780273f, 0.7765238881111145f}},
  {{1.0f, 0.0f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.794854462146759f, -0.6068001389503479f}, {0.829405665397644f, -0.5586467385292053f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.9982437491416931f, -0.05924062803387642f}, {0.3758275806903839f, -0.926689624786377f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.9929810762405396f, 0.11827316880226135f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.7175072431564331f, -0.6965510249137878f}, {0.8896570801734924f, -0.4566292464733124f}, {0.14764656126499176f, 0.989040195941925f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.4827921986579895f, -0.8757349252700806f}, {0.674983024597168f, 0.7378332614898682f}, {-0.9151456356048584f, 0.4031234383583069f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.9720228910446167f, 0.2348860502243042f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.9374196529388428f, -0.3482016324996948f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.956400990486145f, -0.29205676913261414f}, {0.5829795002937317f, -0.8124868869781494f}},
  {{1.0f, 0.0f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.9720228910446167f, -0.2348860502243042f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.794854462146759f, -0.6068001389503479f}, {0.8896570801734924f, -0.4566292464733124f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.9151456356048584f, -0.4031234383583069f}, {0.7575112581253052f, -0.6528221368789673f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.5829795002937317f, -0.8124868869781494f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.9982437491416931f, 0.05924062803387642f}, {0.3758275806903839f, -0.926689624786377f}, {0.674983024597168f, 0.7378332614898682f}, {-0.956400990486145f, 0.29205676913261414f}, {0.14764656126499176f, -0.989040195941925f}, {0.829405665397644f, 0.5586467385292053f}, {-0.8610436320304871f, 0.5085310935974121f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.9374196529388428f, 0.3482016324996948f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.9929810762405396f, 0.11827316880226135f}, {-0.5338233709335327f, 0.8455960154533386f}},
  {{1.0f, 0.0f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.9929810762405396f, 0.11827316880226135f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.9720228910446167f, 0.2348860502243042f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.9374196529388428f, 0.3482016324996948f}, {-0.794854462146759f, 0.6068001389503479f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.8610436320304871f, 0.5085310935974121f}, {0.029633328318595886f, -0.9995608329772949f}, {0.829405665397644f, 0.5586467385292053f}, {-0.9151456356048584f, 0.4031234383583069f}, {0.14764656126499176f, -0.989040195941925f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.956400990486145f, 0.29205676913261414f}, {0.26358717679977417f, -0.9646356105804443f}, {0.674983024597168f, 0.7378332614898682f}, {-0.9842305779457092f, 0.1768902689218521f}, {0.3758275806903839f, -0.926689624786377f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.9982437491416931f, 0.05924062803387642f}, {0.4827921986579895f, -0.8757349252700806f}},
  {{1.0f, 0.0f}, {-0.6300878524780273f, 0.7765238881111145f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.9151456356048584f, 0.4031234383583069f}, {0.26358717679977417f, -0.9646356105804443f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.9982437491416931f, -0.05924062803387642f}, {0.674983024597168f, -0.7378332614898682f}, {0.14764656126499176f, 0.989040195941925f}, {-0.8610436320304871f, -0.5085310935974121f}, {0.9374196529388428f, -0.3482016324996948f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.9929810762405396f, 0.11827316880226135f}, {-0.7175072431564331f, 0.6965510249137878f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.829405665397644f, 0.5586467385292053f}, {-0.956400990486145f, 0.29205676913261414f}, {0.3758275806903839f, -0.926689624786377f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.7575112581253052f, -0.6528221368789673f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.794854462146759f, -0.6068001389503479f}, {0.9720228910446167f, -0.2348860502243042f}, {-0.43006521463394165f, 0.9027978181838989f}},
  {{1.0f, 0.0f}, {-0.7175072431564331f, 0.6965510249137878f}, {0.029633328318595886f, -0.9995608329772949f}, {0.674983024597168f, 0.7378332614898682f}, {-0.9982437491416931f, -0.05924062803387642f}, {0.7575112581253052f, -0.6528221368789673f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.9929810762405396f, 0.11827316880226135f}, {-0.794854462146759f, 0.6068001389503479f}, {0.14764656126499176f, -0.989040195941925f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.829405665397644f, -0.5586467385292053f}, {-0.2059786170721054f, 0.9785565137863159f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.9720228910446167f, 0.2348860502243042f}, {-0.8610436320304871f, 0.5085310935974121f}, {0.26358717679977417f, -0.9646356105804443f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.956400990486145f, -0.29205676913261414f}, {0.8896570801734924f, -0.4566292464733124f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.9374196529388428f, 0.3482016324996948f}, {-0.9151456356048584f, 0.4031234383583069f}, {0.3758275806903839f, -0.926689624786377f}},
  {{1.0f, 0.0f}, {-0.794854462146759f, 0.6068001389503479f}, {0.26358717679977417f, -0.9646356105804443f}, {0.3758275806903839f, 0.926689624786377f}, {-0.8610436320304871f, -0.5085310935974121f}, {0.9929810762405396f, -0.11827316880226135f}, {-0.7175072431564331f, 0.6965510249137878f}, {0.14764656126499176f, -0.989040195941925f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.9151456356048584f, -0.4031234383583069f}, {0.9720228910446167f, -0.2348860502243042f}, {-0.6300878524780273f, 0.7765238881111145f}, {0.029633328318595886f, -0.9995608329772949f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.956400990486145f, -0.29205676913261414f}, {0.9374196529388428f, -0.3482016324996948f}, {-0.5338233709335327f, 0.8455960154533386f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.674983024597168f, 0.7378332614898682f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.8896570801734924f, -0.4566292464733124f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.9982437491416931f, -0.05924062803387642f}, {0.829405665397644f, -0.5586467385292053f}, {-0.3202698528766632f, 0.9473263621330261f}},
  {{1.0f, 0.0f}, {-0.8610436320304871f, 0.5085310935974121f}, {0.4827921986579895f, -0.8757349252700806f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.9982437491416931f, 0.05924062803387642f}, {0.829405665397644f, -0.5586467385292053f}, {-0.43006521463394165f, 0.9027978181838989f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.9151456356048584f, -0.4031234383583069f}, {0.9929810762405396f, -0.11827316880226135f}, {-0.794854462146759f, 0.6068001389503479f}, {0.3758275806903839f, -0.926689624786377f}, {0.14764656126499176f, 0.989040195941925f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.9374196529388428f, 0.3482016324996948f}, {-0.9842305779457092f, 0.1768902689218521f}, {0.7575112581253052f, -0.6528221368789673f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.674983024597168f, 0.7378332614898682f}, {-0.956400990486145f, -0.29205676913261414f}, {0.9720228910446167f, -0.2348860502243042f}, {-0.7175072431564331f, 0.6965510249137878f}, {0.26358717679977417f, -0.9646356105804443f}},
  {{1.0f, 0.0f}, {-0.9151456356048584f, 0.4031234383583069f}, {0.674983024597168f, -0.7378332614898682f}, {-0.3202698528766632f, 0.9473263621330261f}, {-0.08879589289426804f, -0.9960498213768005f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.794854462146759f, -0.6068001389503479f}, {0.9720228910446167f, 0.2348860502243042f}, {-0.9842305779457092f, 0.1768902689218521f}, {0.829405665397644f, -0.5586467385292053f}, {-0.5338233709335327f, 0.8455960154533386f}, {0.14764656126499176f, -0.989040195941925f}, {0.26358717679977417f, 0.9646356105804443f}, {-0.6300878524780273f, -0.7765238881111145f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.9982437491416931f, -0.05924062803387642f}, {0.9374196529388428f, -0.3482016324996948f}, {-0.7175072431564331f, 0.6965510249137878f}, {0.3758275806903839f, -0.926689624786377f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.43006521463394165f, -0.9027978181838989f}, {0.7575112581253052f, 0.6528221368789673f}, {-0.956400990486145f, -0.29205676913261414f}, {0.9929810762405396f, -0.11827316880226135f}, {-0.8610436320304871f, 0.5085310935974121f}, {0.5829795002937317f, -0.8124868869781494f}, {-0.2059786170721054f, 0.9785565137863159f}},
  {{1.0f, 0.0f}, {-0.956400990486145f, 0.29205676913261414f}, {0.829405665397644f, -0.5586467385292053f}, {-0.6300878524780273f, 0.7765238881111145f}, {0.3758275806903839f, -0.926689624786377f}, {-0.08879589289426804f, 0.9960498213768005f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.4827921986579895f, 0.8757349252700806f}, {-0.7175072431564331f, -0.6965510249137878f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.9842305779457092f, -0.1768902689218521f}, {0.9929810762405396f, -0.11827316880226135f}, {-0.9151456356048584f, 0.4031234383583069f}, {0.7575112581253052f, -0.6528221368789673f}, {-0.5338233709335327f, 0.8455960154533386f}, {0.26358717679977417f, -0.9646356105804443f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.3202698528766632f, -0.9473263621330261f}, {0.5829795002937317f, 0.8124868869781494f}, {-0.794854462146759f, -0.6068001389503479f}, {0.9374196529388428f, 0.3482016324996948f}, {-0.9982437491416931f, -0.05924062803387642f}, {0.9720228910446167f, -0.2348860502243042f}, {-0.8610436320304871f, 0.5085310935974121f}, {0.674983024597168f, -0.7378332614898682f}, {-0.43006521463394165f, 0.9027978181838989f}, {0.14764656126499176f, -0.989040195941925f}},
  {{1.0f, 0.0f}, {-0.9842305779457092f, 0.1768902689218521f}, {0.9374196529388428f, -0.3482016324996948f}, {-0.8610436320304871f, 0.5085310935974121f}, {0.7575112581253052f, -0.6528221368789673f}, {-0.6300878524780273f, 0.7765238881111145f}, {0.4827921986579895f, -0.8757349252700806f}, {-0.3202698528766632f, 0.9473263621330261f}, {0.14764656126499176f, -0.989040195941925f}, {0.029633328318595886f, 0.9995608329772949f}, {-0.2059786170721054f, -0.9785565137863159f}, {0.3758275806903839f, 0.926689624786377f}, {-0.5338233709335327f, -0.8455960154533386f}, {0.674983024597168f, 0.7378332614898682f}, {-0.794854462146759f, -0.6068001389503479f}, {0.8896570801734924f, 0.4566292464733124f}, {-0.956400990486145f, -0.29205676913261414f}, {0.9929810762405396f, 0.11827316880226135f}, {-0.9982437491416931f, 0.05924062803387642f}, {0.9720228910446167f, -0.2348860502243042f}, {-0.9151456356048584f, 0.4031234383583069f}, {0.829405665397644f, -0.5586467385292053f}, {-0.7175072431564331f, 0.6965510249137878f}, {0.5829795002937317f, -0.8124868869781494f}, {-0.43006521463394165f, 0.9027978181838989f}, {0.26358717679977417f, -0.9646356105804443f}, {-0.08879589289426804f, 0.9960498213768005f}},
  {{1.0f, 0.0f}, {-0.9982437491416931f, 0.05924062803387642f}, {0.9929810762405396f, -0.11827316880226135f}, {-0.9842305779457092f, 0.1768902689218521f}, {0.9720228910446167f, -0.2348860502243042f}, {-0.956400990486145f, 0.29205676913261414f}, {0.9374196529388428f, -0.3482016324996948f}, {-0.9151456356048584f, 0.4031234383583069f}, {0.8896570801734924f, -0.4566292464733124f}, {-0.8610436320304871f, 0.5085310935974121f}, {0.829405665397644f, -0.5586467385292053f}, {-0.794854462146759f, 0.6068001389503479f}, {0.7575112581253052f, -0.6528221368789673f}, {-0.7175072431564331f, 0.6965510249137878f}, {0.674983024597168f, -0.7378332614898682f}, {-0.6300878524780273f, 0.7765238881111145f}, {0.5829795002937317f, -0.8124868869781494f}, {-0.5338233709335327f, 0.8455960154533386f}, {0.4827921986579895f, -0.8757349252700806f}, {-0.43006521463394165f, 0.9027978181838989f}, {0.3758275806903839f, -0.926689624786377f}, {-0.3202698528766632f, 0.9473263621330261f}, {0.26358717679977417f, -0.9646356105804443f}, {-0.2059786170721054f, 0.9785565137863159f}, {0.14764656126499176f, -0.989040195941925f}, {-0.08879589289426804f, 0.9960498213768005f}, {0.029633328318595886f, -0.9995608329772949f}}};
template <bool INV, bool PAIRED = false, typename St>
__device__ __forceinline__ void dft_r53_compact(const float2* v, St&& st, int kmax = 26) {
  const float2 x0 = v[0];
  const f2reg X0 = f2pk(x0);
  const f2reg S1 = f2add(f2pk(v[1]), f2pk(v[52]));
  const f2reg D1 = f2sub(f2pk(v[1]), f2pk(v[52]));
  const f2reg S2 = f2add(f2pk(v[2]), f2pk(v[51]));
  const f2reg D2 = f2sub(f2pk(v[2]), f2pk(v[51]));
  const f2reg S3 = f2add(f2pk(v[3]), f2pk(v[50]));
  const f2reg D3 = f2sub(f2pk(v[3]), f2pk(v[50]));
  const f2reg S4 = f2add(f2pk(v[4]), f2pk(v[49]));
  const f2reg D4 = f2sub(f2pk(v[4]), f2pk(v[49]));
  const f2reg S5 = f2add(f2pk(v[5]), f2pk(v[48]));
  const f2reg D5 = f2sub(f2pk(v[5]), f2pk(v[48]));
  const f2reg S6 = f2add(f2pk(v[6]), f2pk(v[47]));
  const f2reg D6 = f2sub(f2pk(v[6]), f2pk(v[47]));
  const f2reg S7 = f2add(f2pk(v[7]), f2pk(v[46]));
  const f2reg D7 = f2sub(f2pk(v[7]), f2pk(v[46]));
  const f2reg S8 = f2add(f2pk(v[8]), f2pk(v[45]));
  const f2reg D8 = f2sub(f2pk(v[8]), f2pk(v[45]));
  const f2reg S9 = f2add(f2pk(v[9]), f2pk(v[44]));
  const f2reg D9 = f2sub(f2pk(v[9]), f2pk(v[44]));
  const f2reg S10 = f2add(f2pk(v[10]), f2pk(v[43]));
  const f2reg D10 = f2sub(f2pk(v[10]), f2pk(v[43]));
  const f2reg S11 = f2add(f2pk(v[11]), f2pk(v[42]));
  const f2reg D11 = f2sub(f2pk(v[11]), f2pk(v[42]));
  const f2reg S12 = f2add(f2pk(v[12]), f2pk(v[41]));
  const f2reg D12 = f2sub(f2pk(v[12]), f2pk(v[41]));
  const f2reg S13 = f2add(f2pk(v[13]), f2pk(v[40]));
  const f2reg D13 = f2sub(f2pk(v[13]), f2pk(v[40]));
  const f2reg S14 = f2add(f2pk(v[14]), f2pk(v[39]));
  const f2reg D14 = f2sub(f2pk(v[14]), f2pk(v[39]));
  const f2reg S15 = f2add(f2pk(v[15]), f2pk(v[38]));
  const f2reg D15 = f2sub(f2pk(v[15]), f2pk(v[38]));
  const f2reg S16 = f2add(f2pk(v[16]), f2pk(v[37]));
  const f2reg D16 = f2sub(f2pk(v[16]), f2pk(v[37]));
  const f2reg S17 = f2add(f2pk(v[17]), f2pk(v[36]));
  const f2reg D17 = f2sub(f2pk(v[17]), f2pk(v[36]));
  const f2reg S18 = f2add(f2pk(v[18]), f2pk(v[35]));
  const f2reg D18 = f2sub(f2pk(v[18]), f2pk(v[35]));
  const f2reg S19 = f2add(f2pk(v[19]), f2pk(v[34]));
  const f2reg D19 = f2sub(f2pk(v[19]), f2pk(v[34]));
  const f2reg S20 = f2add(f2pk(v[20]), f2pk(v[33]));
  const f2reg D20 = f2sub(f2pk(v[20]), f2pk(v[33]));
  const f2reg S21 = f2add(f2pk(v[21]), f2pk(v[32]));
  const f2reg D21 = f2sub(f2pk(v[21]), f2pk(v[32]));
  const f2reg S22 = f2add(f2pk(v[22]), f2pk(v[31]));
  const f2reg D22 = f2sub(f2pk(v[22]), f2pk(v[31]));
  const f2reg S23 = f2add(f2pk(v[23]), f2pk(v[30]));
  const f2reg D23 = f2sub(f2pk(v[23]), f2pk(v[30]));
  const f2reg S24 = f2add(f2pk(v[24]), f2pk(v[29]));
  const f2reg D24 = f2sub(f2pk(v[24]), f2pk(v[29]));
  const f2reg S25 = f2add(f2pk(v[25]), f2pk(v[28]));
  const f2reg D25 = f2sub(f2pk(v[25]), f2pk(v[28]));
  const f2reg S26 = f2add(f2pk(v[26]), f2pk(v[27]));
  const f2reg D26 = f2sub(f2pk(v[26]), f2pk(v[27]));
  {
    f2reg t = S1;
    t = f2add(t, S2);
    t = f2add(t, S3);
    t = f2add(t, S4);
    t = f2add(t, S5);
    t = f2add(t, S6);
    t = f2add(t, S7);
    t = f2add(t, S8);
    t = f2add(t, S9);
    t = f2add(t, S10);
    t = f2add(t, S11);
    t = f2add(t, S12);
    t = f2add(t, S13);
    t = f2add(t, S14);
    t = f2add(t, S15);
    t = f2add(t, S16);
    t = f2add(t, S17);
    t = f2add(t, S18);
    t = f2add(t, S19);
    t = f2add(t, S20);
    t = f2add(t, S21);
    t = f2add(t, S22);
    t = f2add(t, S23);
    t = f2add(t, S24);
    t = f2add(t, S25);
    t = f2add(t, S26);
    st(0, f2up(f2add(X0, t)));
  }
  if constexpr (PAIRED) {
#pragma unroll 1
    for (int k = 1; k <= 13; k++) {
      const float2* t = c_tw53[k];
      const float2* u = c_tw53[k + 13];
      f2reg A = X0, B = 0ull, C = X0, E = 0ull;
      { const float2 c = t[1], e = u[1]; A = f2fma(S1, f2splat(c.x), A); B = f2fma(D1, f2splat(c.y), B); C = f2fma(S1, f2splat(e.x), C); E = f2fma(D1, f2splat(e.y), E); }
      { const float2 c = t[2], e = u[2]; A = f2fma(S2, f2splat(c.x), A); B = f2fma(D2, f2splat(c.y), B); C = f2fma(S2, f2splat(e.x), C); E = f2fma(D2, f2splat(e.y), E); }
      { const float2 c = t[3], e = u[3]; A = f2fma(S3, f2splat(c.x), A); B = f2fma(D3, f2splat(c.y), B); C = f2fma(S3, f2splat(e.x), C); E = f2fma(D3, f2splat(e.y), E); }
      { const float2 c = t[4], e = u[4]; A = f2fma(S4, f2splat(c.x), A); B = f2fma(D4, f2splat(c.y), B); C = f2fma(S4, f2splat(e.x), C); E = f2fma(D4, f2splat(e.y), E); }
      { const float2 c = t[5], e = u[5]; A = f2fma(S5, f2splat(c.x), A); B = f2fma(D5, f2splat(c.y), B); C = f2fma(S5, f2splat(e.x), C); E = f2fma(D5, f2splat(e.y), E); }
      { const float2 c = t[6], e = u[6]; A = f2fma(S6, f2splat(c.x), A); B = f2fma(D6, f2splat(c.y), B); C = f2fma(S6, f2splat(e.x), C); E = f2fma(D6, f2splat(e.y), E); }
      { const float2 c = t[7], e = u[7]; A = f2fma(S7, f2splat(c.x), A); B = f2fma(D7, f2splat(c.y), B); C = f2fma(S7, f2splat(e.x), C); E = f2fma(D7, f2splat(e.y), E); }
      { const float2 c = t[8], e = u[8]; A = f2fma(S8, f2splat(c.x), A); B = f2fma(D8, f2splat(c.y), B); C = f2fma(S8, f2splat(e.x), C); E = f2fma(D8, f2splat(e.y), E); }
      { const float2 c = t[9], e = u[9]; A = f2fma(S9, f2splat(c.x), A); B = f2fma(D9, f2splat(c.y), B); C = f2fma(S9, f2splat(e.x), C); E = f2fma(D9, f2splat(e.y), E); }
      { const float2 c = t[10], e = u[10]; A = f2fma(S10, f2splat(c.x), A); B = f2fma(D10, f2splat(c.y), B); C = f2fma(S10, f2splat(e.x), C); E = f2fma(D10, f2splat(e.y), E); }
      { const float2 c = t[11], e = u[11]; A = f2fma(S11, f2splat(c.x), A); B = f2fma(D11, f2splat(c.y), B); C = f2fma(S11, f2splat(e.x), C); E = f2fma(D11, f2splat(e.y), E); }
      { const float2 c = t[12], e = u[12]; A = f2fma(S12, f2splat(c.x), A); B = f2fma(D12, f2splat(c.y), B); C = f2fma(S12, f2splat(e.x), C); E = f2fma(D12, f2splat(e.y), E); }
      { const float2 c = t[13], e = u[13]; A = f2fma(S13, f2splat(c.x), A); B = f2fma(D13, f2splat(c.y), B); C = f2fma(S13, f2splat(e.x), C); E = f2fma(D13, f2splat(e.y), E); }
      { const float2 c = t[14], e = u[14]; A = f2fma(S14, f2splat(c.x), A); B = f2fma(D14, f2splat(c.y), B); C = f2fma(S14, f2splat(e.x), C); E = f2fma(D14, f2splat(e.y), E); }
      { const float2 c = t[15], e = u[15]; A = f2fma(S15, f2splat(c.x), A); B = f2fma(D15, f2splat(c.y), B); C = f2fma(S15, f2splat(e.x), C); E = f2fma(D15, f2splat(e.y), E); }
      { const float2 c = t[16], e = u[16]; A = f2fma(S16, f2splat(c.x), A); B = f2fma(D16, f2splat(c.y), B); C = f2fma(S16, f2splat(e.x), C); E = f2fma(D16, f2splat(e.y), E); }
      { const float2 c = t[17], e = u[17]; A = f2fma(S17, f2splat(c.x), A); B = f2fma(D17, f2splat(c.y), B); C = f2fma(S17, f2splat(e.x), C); E = f2fma(D17, f2splat(e.y), E); }
      { const float2 c = t[18], e = u[18]; A = f2fma(S18, f2splat(c.x), A); B = f2fma(D18, f2splat(c.y), B); C = f2fma(S18, f2splat(e.x), C); E = f2fma(D18, f2splat(e.y), E); }
      { const float2 c = t[19], e = u[19]; A = f2fma(S19, f2splat(c.x), A); B = f2fma(D19, f2splat(c.y), B); C = f2fma(S19, f2splat(e.x), C); E = f2fma(D19, f2splat(e.y), E); }
      { const float2 c = t[20], e = u[20]; A = f2fma(S20, f2splat(c.x), A); B = f2fma(D20, f2splat(c.y), B); C = f2fma(S20, f2splat(e.x), C); E = f2fma(D20, f2splat(e.y), E); }
      { const float2 c = t[21], e = u[21]; A = f2fma(S21, f2splat(c.x), A); B = f2fma(D21, f2splat(c.y), B); C = f2fma(S21, f2splat(e.x), C); E = f2fma(D21, f2splat(e.y), E); }
      { const float2 c = t[22], e = u[22]; A = f2fma(S22, f2splat(c.x), A); B = f2fma(D22, f2splat(c.y), B); C = f2fma(S22, f2splat(e.x), C); E = f2fma(D22, f2splat(e.y), E); }
      { const float2 c = t[23], e = u[23]; A = f2fma(S23, f2splat(c.x), A); B = f2fma(D23, f2splat(c.y), B); C = f2fma(S23, f2splat(e.x), C); E = f2fma(D23, f2splat(e.y), E); }
      { const float2 c = t[24], e = u[24]; A = f2fma(S24, f2splat(c.x), A); B = f2fma(D24, f2splat(c.y), B); C = f2fma(S24, f2splat(e.x), C); E = f2fma(D24, f2splat(e.y), E); }
      { const float2 c = t[25], e = u[25]; A = f2fma(S25, f2splat(c.x), A); B = f2fma(D25, f2splat(c.y), B); C = f2fma(S25, f2splat(e.x), C); E = f2fma(D25, f2splat(e.y), E); }
      { const float2 c = t[26], e = u[26]; A = f2fma(S26, f2splat(c.x), A); B = f2fma(D26, f2splat(c.y), B); C = f2fma(S26, f2splat(e.x), C); E = f2fma(D26, f2splat(e.y), E); }
      { const float2 a = f2up(A), b = f2up(B);
        if (!INV) { st(k, make_float2(a.x + b.y, a.y - b.x)); st(53 - (k), make_float2(a.x - b.y, a.y + b.x)); }
        else { st(k, make_float2(a.x - b.y, a.y + b.x)); st(53 - (k), make_float2(a.x + b.y, a.y - b.x)); } }
      { const float2 a = f2up(C), b = f2up(E);
        if (!INV) { st(k + 13, make_float2(a.x + b.y, a.y - b.x)); st(53 - (k + 13), make_float2(a.x - b.y, a.y + b.x)); }
        else { st(k + 13, make_float2(a.x - b.y, a.y + b.x)); st(53 - (k + 13), make_float2(a.x + b.y, a.y - b.x)); } }
    }
  } else {
#pragma unroll 1
    for (int k = 1; k <= kmax; k++) {
      const float2* t = c_tw53[k];
      f2reg A = X0, B = 0ull;
      { const float2 c = t[1]; A = f2fma(S1, f2splat(c.x), A); B = f2fma(D1, f2splat(c.y), B); }
      { const float2 c = t[2]; A = f2fma(S2, f2splat(c.x), A); B = f2fma(D2, f2splat(c.y), B); }
      { const float2 c = t[3]; A = f2fma(S3, f2splat(c.x), A); B = f2fma(D3, f2splat(c.y), B); }
      { const float2 c = t[4]; A = f2fma(S4, f2splat(c.x), A); B = f2fma(D4, f2splat(c.y), B); }
      { const float2 c = t[5]; A = f2fma(S5, f2splat(c.x), A); B = f2fma(D5, f2splat(c.y), B); }
      { const float2 c = t[6]; A = f2fma(S6, f2splat(c.x), A); B = f2fma(D6, f2splat(c.y), B); }
      { const float2 c = t[7]; A = f2fma(S7, f2splat(c.x), A); B = f2fma(D7, f2splat(c.y), B); }
      { const float2 c = t[8]; A = f2fma(S8, f2splat(c.x), A); B = f2fma(D8, f2splat(c.y), B); }
      { const float2 c = t[9]; A = f2fma(S9, f2splat(c.x), A); B = f2fma(D9, f2splat(c.y), B); }
      { const float2 c = t[10]; A = f2fma(S10, f2splat(c.x), A); B = f2fma(D10, f2splat(c.y), B); }
      { const float2 c = t[11]; A = f2fma(S11, f2splat(c.x), A); B = f2fma(D11, f2splat(c.y), B); }
      { const float2 c = t[12]; A = f2fma(S12, f2splat(c.x), A); B = f2fma(D12, f2splat(c.y), B); }
      { const float2 c = t[13]; A = f2fma(S13, f2splat(c.x), A); B = f2fma(D13, f2splat(c.y), B); }
      { const float2 c = t[14]; A = f2fma(S14, f2splat(c.x), A); B = f2fma(D14, f2splat(c.y), B); }
      { const float2 c = t[15]; A = f2fma(S15, f2splat(c.x), A); B = f2fma(D15, f2splat(c.y), B); }
      { const float2 c = t[16]; A = f2fma(S16, f2splat(c.x), A); B = f2fma(D16, f2splat(c.y), B); }
      { const float2 c = t[17]; A = f2fma(S17, f2splat(c.x), A); B = f2fma(D17, f2splat(c.y), B); }
      { const float2 c = t[18]; A = f2fma(S18, f2splat(c.x), A); B = f2fma(D18, f2splat(c.y), B); }
      { const float2 c = t[19]; A = f2fma(S19, f2splat(c.x), A); B = f2fma(D19, f2splat(c.y), B); }
      { const float2 c = t[20]; A = f2fma(S20, f2splat(c.x), A); B = f2fma(D20, f2splat(c.y), B); }
      { const float2 c = t[21]; A = f2fma(S21, f2splat(c.x), A); B = f2fma(D21, f2splat(c.y), B); }
      { const float2 c = t[22]; A = f2fma(S22, f2splat(c.x), A); B = f2fma(D22, f2splat(c.y), B); }
      { const float2 c = t[23]; A = f2fma(S23, f2splat(c.x), A); B = f2fma(D23, f2splat(c.y), B); }
      { const float2 c = t[24]; A = f2fma(S24, f2splat(c.x), A); B = f2fma(D24, f2splat(c.y), B); }
      { const float2 c = t[25]; A = f2fma(S25, f2splat(c.x), A); B = f2fma(D25, f2splat(c.y), B); }
      { const float2 c = t[26]; A = f2fma(S26, f2splat(c.x), A); B = f2fma(D26, f2splat(c.y), B); }
      { const float2 a = f2up(A), b = f2up(B);
        if (!INV) { st(k, make_float2(a.x + b.y, a.y - b.x)); st(53 - (k), make_float2(a.x - b.y, a.y + b.x)); }
        else { st(k, make_float2(a.x - b.y, a.y + b.x)); st(53 - (k), make_float2(a.x + b.y, a.y - b.x)); } }
    }
  }
}
}  // namespace mc
