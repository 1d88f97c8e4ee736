// Generated by gen_dft.py -- do not edit by hand.
// Straight-line odd-radix DFT butterflies (symmetric direct form).
#pragma once
#include <cuda_runtime.h>
namespace mc {
constexpr int kGeneratedOddRadices[] = {3, 5, 7, 11, 13, 53};
template <bool INV> __device__ __forceinline__ void dft_r3(float2* v) {
  const float2 x0 = v[0];
  const float2 s1 = make_float2(v[1].x + v[2].x, v[1].y + v[2].y);
  const float2 d1 = make_float2(v[1].x - v[2].x, v[1].y - v[2].y);
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
}
template <bool INV> __device__ __forceinline__ void dft_r5(float2* v) {
  const float2 x0 = v[0];
  const float2 s1 = make_float2(v[1].x + v[4].x, v[1].y + v[4].y);
  const float2 d1 = make_float2(v[1].x - v[4].x, v[1].y - v[4].y);
  const float2 s2 = make_float2(v[2].x + v[3].x, v[2].y + v[3].y);
  const float2 d2 = make_float2(v[2].x - v[3].x, v[2].y - v[3].y);
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
}
template <bool INV> __device__ __forceinline__ void dft_r7(float2* v) {
  const float2 x0 = v[0];
  const float2 s1 = make_float2(v[1].x + v[6].x, v[1].y + v[6].y);
  const float2 d1 = make_float2(v[1].x - v[6].x, v[1].y - v[6].y);
  const float2 s2 = make_float2(v[2].x + v[5].x, v[2].y + v[5].y);
  const float2 d2 = make_float2(v[2].x - v[5].x, v[2].y - v[5].y);
  const float2 s3 = make_float2(v[3].x + v[4].x, v[3].y + v[4].y);
  const float2 d3 = make_float2(v[3].x - v[4].x, v[3].y - v[4].y);
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
}
template <bool INV> __device__ __forceinline__ void dft_r11(float2* v) {
  const float2 x0 = v[0];
  const float2 s1 = make_float2(v[1].x + v[10].x, v[1].y + v[10].y);
  const float2 d1 = make_float2(v[1].x - v[10].x, v[1].y - v[10].y);
  const float2 s2 = make_float2(v[2].x + v[9].x, v[2].y + v[9].y);
  const float2 d2 = make_float2(v[2].x - v[9].x, v[2].y - v[9].y);
  const float2 s3 = make_float2(v[3].x + v[8].x, v[3].y + v[8].y);
  const float2 d3 = make_float2(v[3].x - v[8].x, v[3].y - v[8].y);
  const float2 s4 = make_float2(v[4].x + v[7].x, v[4].y + v[7].y);
  const float2 d4 = make_float2(v[4].x - v[7].x, v[4].y - v[7].y);
  const float2 s5 = make_float2(v[5].x + v[6].x, v[5].y + v[6].y);
  const float2 d5 = make_float2(v[5].x - v[6].x, v[5].y - v[6].y);
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
}
template <bool INV> __device__ __forceinline__ void dft_r13(float2* v) {
  const float2 x0 = v[0];
  const float2 s1 = make_float2(v[1].x + v[12].x, v[1].y + v[12].y);
  const float2 d1 = make_float2(v[1].x - v[12].x, v[1].y - v[12].y);
  const float2 s2 = make_float2(v[2].x + v[11].x, v[2].y + v[11].y);
  const float2 d2 = make_float2(v[2].x - v[11].x, v[2].y - v[11].y);
  const float2 s3 = make_float2(v[3].x + v[10].x, v[3].y + v[10].y);
  const float2 d3 = make_float2(v[3].x - v[10].x, v[3].y - v[10].y);
  const float2 s4 = make_float2(v[4].x + v[9].x, v[4].y + v[9].y);
  const float2 d4 = make_float2(v[4].x - v[9].x, v[4].y - v[9].y);
  const float2 s5 = make_float2(v[5].x + v[8].x, v[5].y + v[8].y);
  const float2 d5 = make_float2(v[5].x - v[8].x, v[5].y - v[8].y);
  const float2 s6 = make_float2(v[6].x + v[7].x, v[6].y + v[7].y);
  const float2 d6 = make_float2(v[6].x - v[7].x, v[6].y - v[7].y);
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
}
template <bool INV> __device__ __forceinline__ void dft_r53(float2* v) {
  const float2 x0 = v[0];
  const float2 s1 = make_float2(v[1].x + v[52].x, v[1].y + v[52].y);
  const float2 d1 = make_float2(v[1].x - v[52].x, v[1].y - v[52].y);
  const float2 s2 = make_float2(v[2].x + v[51].x, v[2].y + v[51].y);
  const float2 d2 = make_float2(v[2].x - v[51].x, v[2].y - v[51].y);
  const float2 s3 = make_float2(v[3].x + v[50].x, v[3].y + v[50].y);
  const float2 d3 = make_float2(v[3].x - v[50].x, v[3].y - v[50].y);
  const float2 s4 = make_float2(v[4].x + v[49].x, v[4].y + v[49].y);
  const float2 d4 = make_float2(v[4].x - v[49].x, v[4].y - v[49].y);
  const float2 s5 = make_float2(v[5].x + v[48].x, v[5].y + v[48].y);
  const float2 d5 = make_float2(v[5].x - v[48].x, v[5].y - v[48].y);
  const float2 s6 = make_float2(v[6].x + v[47].x, v[6].y + v[47].y);
  const float2 d6 = make_float2(v[6].x - v[47].x, v[6].y - v[47].y);
  const float2 s7 = make_float2(v[7].x + v[46].x, v[7].y + v[46].y);
  const float2 d7 = make_float2(v[7].x - v[46].x, v[7].y - v[46].y);
  const float2 s8 = make_float2(v[8].x + v[45].x, v[8].y + v[45].y);
  const float2 d8 = make_float2(v[8].x - v[45].x, v[8].y - v[45].y);
  const float2 s9 = make_float2(v[9].x + v[44].x, v[9].y + v[44].y);
  const float2 d9 = make_float2(v[9].x - v[44].x, v[9].y - v[44].y);
  const float2 s10 = make_float2(v[10].x + v[43].x, v[10].y + v[43].y);
  const float2 d10 = make_float2(v[10].x - v[43].x, v[10].y - v[43].y);
  const float2 s11 = make_float2(v[11].x + v[42].x, v[11].y + v[42].y);
  const float2 d11 = make_float2(v[11].x - v[42].x, v[11].y - v[42].y);
  const float2 s12 = make_float2(v[12].x + v[41].x, v[12].y + v[41].y);
  const float2 d12 = make_float2(v[12].x - v[41].x, v[12].y - v[41].y);
  const float2 s13 = make_float2(v[13].x + v[40].x, v[13].y + v[40].y);
  const float2 d13 = make_float2(v[13].x - v[40].x, v[13].y - v[40].y);
  const float2 s14 = make_float2(v[14].x + v[39].x, v[14].y + v[39].y);
  const float2 d14 = make_float2(v[14].x - v[39].x, v[14].y - v[39].y);
  const float2 s15 = make_float2(v[15].x + v[38].x, v[15].y + v[38].y);
  const float2 d15 = make_float2(v[15].x - v[38].x, v[15].y - v[38].y);
  const float2 s16 = make_float2(v[16].x + v[37].x, v[16].y + v[37].y);
  const float2 d16 = make_float2(v[16].x - v[37].x, v[16].y - v[37].y);
  const float2 s17 = make_float2(v[17].x + v[36].x, v[17].y + v[36].y);
  const float2 d17 = make_float2(v[17].x - v[36].x, v[17].y - v[36].y);
  const float2 s18 = make_float2(v[18].x + v[35].x, v[18].y + v[35].y);
  const float2 d18 = make_float2(v[18].x - v[35].x, v[18].y - v[35].y);
  const float2 s19 = make_float2(v[19].x + v[34].x, v[19].y + v[34].y);
  const float2 d19 = make_float2(v[19].x - v[34].x, v[19].y - v[34].y);
  const float2 s20 = make_float2(v[20].x + v[33].x, v[20].y + v[33].y);
  const float2 d20 = make_float2(v[20].x - v[33].x, v[20].y - v[33].y);
  const float2 s21 = make_float2(v[21].x + v[32].x, v[21].y + v[32].y);
  const float2 d21 = make_float2(v[21].x - v[32].x, v[21].y - v[32].y);
  const float2 s22 = make_float2(v[22].x + v[31].x, v[22].y + v[31].y);
  const float2 d22 = make_float2(v[22].x - v[31].x, v[22].y - v[31].y);
  const float2 s23 = make_float2(v[23].x + v[30].x, v[23].y + v[30].y);
  const float2 d23 = make_float2(v[23].x - v[30].x, v[23].y - v[30].y);
  const float2 s24 = make_float2(v[24].x + v[29].x, v[24].y + v[29].y);
  const float2 d24 = make_float2(v[24].x - v[29].x, v[24].y - v[29].y);
  const float2 s25 = make_float2(v[25].x + v[28].x, v[25].y + v[28].y);
  const float2 d25 = make_float2(v[25].x - v[28].x, v[25].y - v[28].y);
  const float2 s26 = make_float2(v[26].x + v[27].x, v[26].y + v[27].y);
  const float2 d26 = make_float2(v[26].x - v[27].x, v[26].y - v[27].y);
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
  const float2 s1 = make_float2(v[1].x + v[52].x, v[1].y + v[52].y);
  const float2 d1 = make_float2(v[1].x - v[52].x, v[1].y - v[52].y);
  const float2 s2 = make_float2(v[2].x + v[51].x, v[2].y + v[51].y);
  const float2 d2 = make_float2(v[2].x - v[51].x, v[2].y - v[51].y);
  const float2 s3 = make_float2(v[3].x + v[50].x, v[3].y + v[50].y);
  const float2 d3 = make_float2(v[3].x - v[50].x, v[3].y - v[50].y);
  const float2 s4 = make_float2(v[4].x + v[49].x, v[4].y + v[49].y);
  const float2 d4 = make_float2(v[4].x - v[49].x, v[4].y - v[49].y);
  const float2 s5 = make_float2(v[5].x + v[48].x, v[5].y + v[48].y);
  const float2 d5 = make_float2(v[5].x - v[48].x, v[5].y - v[48].y);
  const float2 s6 = make_float2(v[6].x + v[47].x, v[6].y + v[47].y);
  const float2 d6 = make_float2(v[6].x - v[47].x, v[6].y - v[47].y);
  const float2 s7 = make_float2(v[7].x + v[46].x, v[7].y + v[46].y);
  const float2 d7 = make_float2(v[7].x - v[46].x, v[7].y - v[46].y);
  const float2 s8 = make_float2(v[8].x + v[45].x, v[8].y + v[45].y);
  const float2 d8 = make_float2(v[8].x - v[45].x, v[8].y - v[45].y);
  const float2 s9 = make_float2(v[9].x + v[44].x, v[9].y + v[44].y);
  const float2 d9 = make_float2(v[9].x - v[44].x, v[9].y - v[44].y);
  const float2 s10 = make_float2(v[10].x + v[43].x, v[10].y + v[43].y);
  const float2 d10 = make_float2(v[10].x - v[43].x, v[10].y - v[43].y);
  const float2 s11 = make_float2(v[11].x + v[42].x, v[11].y + v[42].y);
  const float2 d11 = make_float2(v[11].x - v[42].x, v[11].y - v[42].y);
  const float2 s12 = make_float2(v[12].x + v[41].x, v[12].y + v[41].y);
  const float2 d12 = make_float2(v[12].x - v[41].x, v[12].y - v[41].y);
  const float2 s13 = make_float2(v[13].x + v[40].x, v[13].y + v[40].y);
  const float2 d13 = make_float2(v[13].x - v[40].x, v[13].y - v[40].y);
  const float2 s14 = make_float2(v[14].x + v[39].x, v[14].y + v[39].y);
  const float2 d14 = make_float2(v[14].x - v[39].x, v[14].y - v[39].y);
  const float2 s15 = make_float2(v[15].x + v[38].x, v[15].y + v[38].y);
  const float2 d15 = make_float2(v[15].x - v[38].x, v[15].y - v[38].y);
  const float2 s16 = make_float2(v[16].x + v[37].x, v[16].y + v[37].y);
  const float2 d16 = make_float2(v[16].x - v[37].x, v[16].y - v[37].y);
  const float2 s17 = make_float2(v[17].x + v[36].x, v[17].y + v[36].y);
  const float2 d17 = make_float2(v[17].x - v[36].x, v[17].y - v[36].y);
  const float2 s18 = make_float2(v[18].x + v[35].x, v[18].y + v[35].y);
  const float2 d18 = make_float2(v[18].x - v[35].x, v[18].y - v[35].y);
  const float2 s19 = make_float2(v[19].x + v[34].x, v[19].y + v[34].y);
  const float2 d19 = make_float2(v[19].x - v[34].x, v[19].y - v[34].y);
  const float2 s20 = make_float2(v[20].x + v[33].x, v[20].y + v[33].y);
  const float2 d20 = make_float2(v[20].x - v[33].x, v[20].y - v[33].y);
  const float2 s21 = make_float2(v[21].x + v[32].x, v[21].y + v[32].y);
  const float2 d21 = make_float2(v[21].x - v[32].x, v[21].y - v[32].y);
  const float2 s22 = make_float2(v[22].x + v[31].x, v[22].y + v[31].y);
  const float2 d22 = make_float2(v[22].x - v[31].x, v[22].y - v[31].y);
  const float2 s23 = make_float2(v[23].x + v[30].x, v[23].y + v[30].y);
  const float2 d23 = make_float2(v[23].x - v[30].x, v[23].y - v[30].y);
  const float2 s24 = make_float2(v[24].x + v[29].x, v[24].y + v[29].y);
  const float2 d24 = make_float2(v[24].x - v[29].x, v[24].y - v[29].y);
  const float2 s25 = make_float2(v[25].x + v[28].x, v[25].y + v[28].y);
  const float2 d25 = make_float2(v[25].x - v[28].x, v[25].y - v[28].y);
  const float2 s26 = make_float2(v[26].x + v[27].x, v[26].y + v[27].y);
  const float2 d26 = make_float2(v[26].x - v[27].x, v[26].y - v[27].y);
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
__device__ __forceinline__ void dft_r53_compact(const float2* v, St&& st) {
  const float2 x0 = v[0];
  const float2 s1 = make_float2(v[1].x + v[52].x, v[1].y + v[52].y);
  const float2 d1 = make_float2(v[1].x - v[52].x, v[1].y - v[52].y);
  const float2 s2 = make_float2(v[2].x + v[51].x, v[2].y + v[51].y);
  const float2 d2 = make_float2(v[2].x - v[51].x, v[2].y - v[51].y);
  const float2 s3 = make_float2(v[3].x + v[50].x, v[3].y + v[50].y);
  const float2 d3 = make_float2(v[3].x - v[50].x, v[3].y - v[50].y);
  const float2 s4 = make_float2(v[4].x + v[49].x, v[4].y + v[49].y);
  const float2 d4 = make_float2(v[4].x - v[49].x, v[4].y - v[49].y);
  const float2 s5 = make_float2(v[5].x + v[48].x, v[5].y + v[48].y);
  const float2 d5 = make_float2(v[5].x - v[48].x, v[5].y - v[48].y);
  const float2 s6 = make_float2(v[6].x + v[47].x, v[6].y + v[47].y);
  const float2 d6 = make_float2(v[6].x - v[47].x, v[6].y - v[47].y);
  const float2 s7 = make_float2(v[7].x + v[46].x, v[7].y + v[46].y);
  const float2 d7 = make_float2(v[7].x - v[46].x, v[7].y - v[46].y);
  const float2 s8 = make_float2(v[8].x + v[45].x, v[8].y + v[45].y);
  const float2 d8 = make_float2(v[8].x - v[45].x, v[8].y - v[45].y);
  const float2 s9 = make_float2(v[9].x + v[44].x, v[9].y + v[44].y);
  const float2 d9 = make_float2(v[9].x - v[44].x, v[9].y - v[44].y);
  const float2 s10 = make_float2(v[10].x + v[43].x, v[10].y + v[43].y);
  const float2 d10 = make_float2(v[10].x - v[43].x, v[10].y - v[43].y);
  const float2 s11 = make_float2(v[11].x + v[42].x, v[11].y + v[42].y);
  const float2 d11 = make_float2(v[11].x - v[42].x, v[11].y - v[42].y);
  const float2 s12 = make_float2(v[12].x + v[41].x, v[12].y + v[41].y);
  const float2 d12 = make_float2(v[12].x - v[41].x, v[12].y - v[41].y);
  const float2 s13 = make_float2(v[13].x + v[40].x, v[13].y + v[40].y);
  const float2 d13 = make_float2(v[13].x - v[40].x, v[13].y - v[40].y);
  const float2 s14 = make_float2(v[14].x + v[39].x, v[14].y + v[39].y);
  const float2 d14 = make_float2(v[14].x - v[39].x, v[14].y - v[39].y);
  const float2 s15 = make_float2(v[15].x + v[38].x, v[15].y + v[38].y);
  const float2 d15 = make_float2(v[15].x - v[38].x, v[15].y - v[38].y);
  const float2 s16 = make_float2(v[16].x + v[37].x, v[16].y + v[37].y);
  const float2 d16 = make_float2(v[16].x - v[37].x, v[16].y - v[37].y);
  const float2 s17 = make_float2(v[17].x + v[36].x, v[17].y + v[36].y);
  const float2 d17 = make_float2(v[17].x - v[36].x, v[17].y - v[36].y);
  const float2 s18 = make_float2(v[18].x + v[35].x, v[18].y + v[35].y);
  const float2 d18 = make_float2(v[18].x - v[35].x, v[18].y - v[35].y);
  const float2 s19 = make_float2(v[19].x + v[34].x, v[19].y + v[34].y);
  const float2 d19 = make_float2(v[19].x - v[34].x, v[19].y - v[34].y);
  const float2 s20 = make_float2(v[20].x + v[33].x, v[20].y + v[33].y);
  const float2 d20 = make_float2(v[20].x - v[33].x, v[20].y - v[33].y);
  const float2 s21 = make_float2(v[21].x + v[32].x, v[21].y + v[32].y);
  const float2 d21 = make_float2(v[21].x - v[32].x, v[21].y - v[32].y);
  const float2 s22 = make_float2(v[22].x + v[31].x, v[22].y + v[31].y);
  const float2 d22 = make_float2(v[22].x - v[31].x, v[22].y - v[31].y);
  const float2 s23 = make_float2(v[23].x + v[30].x, v[23].y + v[30].y);
  const float2 d23 = make_float2(v[23].x - v[30].x, v[23].y - v[30].y);
  const float2 s24 = make_float2(v[24].x + v[29].x, v[24].y + v[29].y);
  const float2 d24 = make_float2(v[24].x - v[29].x, v[24].y - v[29].y);
  const float2 s25 = make_float2(v[25].x + v[28].x, v[25].y + v[28].y);
  const float2 d25 = make_float2(v[25].x - v[28].x, v[25].y - v[28].y);
  const float2 s26 = make_float2(v[26].x + v[27].x, v[26].y + v[27].y);
  const float2 d26 = make_float2(v[26].x - v[27].x, v[26].y - v[27].y);
  st(0, make_float2(x0.x + (s1.x + s2.x + s3.x + s4.x + s5.x + s6.x + s7.x + s8.x + s9.x + s10.x + s11.x + s12.x + s13.x + s14.x + s15.x + s16.x + s17.x + s18.x + s19.x + s20.x + s21.x + s22.x + s23.x + s24.x + s25.x + s26.x), x0.y + (s1.y + s2.y + s3.y + s4.y + s5.y + s6.y + s7.y + s8.y + s9.y + s10.y + s11.y + s12.y + s13.y + s14.y + s15.y + s16.y + s17.y + s18.y + s19.y + s20.y + s21.y + s22.y + s23.y + s24.y + s25.y + s26.y)));
  if constexpr (PAIRED) {
#pragma unroll 1
    for (int k = 1; k <= 13; k++) {
      const float2* t = c_tw53[k];
      const float2* u = c_tw53[k + 13];
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      float cr = x0.x, ci = x0.y, dr = 0.0f, di = 0.0f;
      { const float2 c = t[1], e = u[1]; ar = fmaf(s1.x, c.x, ar); ai = fmaf(s1.y, c.x, ai); br = fmaf(d1.x, c.y, br); bi = fmaf(d1.y, c.y, bi); cr = fmaf(s1.x, e.x, cr); ci = fmaf(s1.y, e.x, ci); dr = fmaf(d1.x, e.y, dr); di = fmaf(d1.y, e.y, di); }
      { const float2 c = t[2], e = u[2]; ar = fmaf(s2.x, c.x, ar); ai = fmaf(s2.y, c.x, ai); br = fmaf(d2.x, c.y, br); bi = fmaf(d2.y, c.y, bi); cr = fmaf(s2.x, e.x, cr); ci = fmaf(s2.y, e.x, ci); dr = fmaf(d2.x, e.y, dr); di = fmaf(d2.y, e.y, di); }
      { const float2 c = t[3], e = u[3]; ar = fmaf(s3.x, c.x, ar); ai = fmaf(s3.y, c.x, ai); br = fmaf(d3.x, c.y, br); bi = fmaf(d3.y, c.y, bi); cr = fmaf(s3.x, e.x, cr); ci = fmaf(s3.y, e.x, ci); dr = fmaf(d3.x, e.y, dr); di = fmaf(d3.y, e.y, di); }
      { const float2 c = t[4], e = u[4]; ar = fmaf(s4.x, c.x, ar); ai = fmaf(s4.y, c.x, ai); br = fmaf(d4.x, c.y, br); bi = fmaf(d4.y, c.y, bi); cr = fmaf(s4.x, e.x, cr); ci = fmaf(s4.y, e.x, ci); dr = fmaf(d4.x, e.y, dr); di = fmaf(d4.y, e.y, di); }
      { const float2 c = t[5], e = u[5]; ar = fmaf(s5.x, c.x, ar); ai = fmaf(s5.y, c.x, ai); br = fmaf(d5.x, c.y, br); bi = fmaf(d5.y, c.y, bi); cr = fmaf(s5.x, e.x, cr); ci = fmaf(s5.y, e.x, ci); dr = fmaf(d5.x, e.y, dr); di = fmaf(d5.y, e.y, di); }
      { const float2 c = t[6], e = u[6]; ar = fmaf(s6.x, c.x, ar); ai = fmaf(s6.y, c.x, ai); br = fmaf(d6.x, c.y, br); bi = fmaf(d6.y, c.y, bi); cr = fmaf(s6.x, e.x, cr); ci = fmaf(s6.y, e.x, ci); dr = fmaf(d6.x, e.y, dr); di = fmaf(d6.y, e.y, di); }
      { const float2 c = t[7], e = u[7]; ar = fmaf(s7.x, c.x, ar); ai = fmaf(s7.y, c.x, ai); br = fmaf(d7.x, c.y, br); bi = fmaf(d7.y, c.y, bi); cr = fmaf(s7.x, e.x, cr); ci = fmaf(s7.y, e.x, ci); dr = fmaf(d7.x, e.y, dr); di = fmaf(d7.y, e.y, di); }
      { const float2 c = t[8], e = u[8]; ar = fmaf(s8.x, c.x, ar); ai = fmaf(s8.y, c.x, ai); br = fmaf(d8.x, c.y, br); bi = fmaf(d8.y, c.y, bi); cr = fmaf(s8.x, e.x, cr); ci = fmaf(s8.y, e.x, ci); dr = fmaf(d8.x, e.y, dr); di = fmaf(d8.y, e.y, di); }
      { const float2 c = t[9], e = u[9]; ar = fmaf(s9.x, c.x, ar); ai = fmaf(s9.y, c.x, ai); br = fmaf(d9.x, c.y, br); bi = fmaf(d9.y, c.y, bi); cr = fmaf(s9.x, e.x, cr); ci = fmaf(s9.y, e.x, ci); dr = fmaf(d9.x, e.y, dr); di = fmaf(d9.y, e.y, di); }
      { const float2 c = t[10], e = u[10]; ar = fmaf(s10.x, c.x, ar); ai = fmaf(s10.y, c.x, ai); br = fmaf(d10.x, c.y, br); bi = fmaf(d10.y, c.y, bi); cr = fmaf(s10.x, e.x, cr); ci = fmaf(s10.y, e.x, ci); dr = fmaf(d10.x, e.y, dr); di = fmaf(d10.y, e.y, di); }
      { const float2 c = t[11], e = u[11]; ar = fmaf(s11.x, c.x, ar); ai = fmaf(s11.y, c.x, ai); br = fmaf(d11.x, c.y, br); bi = fmaf(d11.y, c.y, bi); cr = fmaf(s11.x, e.x, cr); ci = fmaf(s11.y, e.x, ci); dr = fmaf(d11.x, e.y, dr); di = fmaf(d11.y, e.y, di); }
      { const float2 c = t[12], e = u[12]; ar = fmaf(s12.x, c.x, ar); ai = fmaf(s12.y, c.x, ai); br = fmaf(d12.x, c.y, br); bi = fmaf(d12.y, c.y, bi); cr = fmaf(s12.x, e.x, cr); ci = fmaf(s12.y, e.x, ci); dr = fmaf(d12.x, e.y, dr); di = fmaf(d12.y, e.y, di); }
      { const float2 c = t[13], e = u[13]; ar = fmaf(s13.x, c.x, ar); ai = fmaf(s13.y, c.x, ai); br = fmaf(d13.x, c.y, br); bi = fmaf(d13.y, c.y, bi); cr = fmaf(s13.x, e.x, cr); ci = fmaf(s13.y, e.x, ci); dr = fmaf(d13.x, e.y, dr); di = fmaf(d13.y, e.y, di); }
      { const float2 c = t[14], e = u[14]; ar = fmaf(s14.x, c.x, ar); ai = fmaf(s14.y, c.x, ai); br = fmaf(d14.x, c.y, br); bi = fmaf(d14.y, c.y, bi); cr = fmaf(s14.x, e.x, cr); ci = fmaf(s14.y, e.x, ci); dr = fmaf(d14.x, e.y, dr); di = fmaf(d14.y, e.y, di); }
      { const float2 c = t[15], e = u[15]; ar = fmaf(s15.x, c.x, ar); ai = fmaf(s15.y, c.x, ai); br = fmaf(d15.x, c.y, br); bi = fmaf(d15.y, c.y, bi); cr = fmaf(s15.x, e.x, cr); ci = fmaf(s15.y, e.x, ci); dr = fmaf(d15.x, e.y, dr); di = fmaf(d15.y, e.y, di); }
      { const float2 c = t[16], e = u[16]; ar = fmaf(s16.x, c.x, ar); ai = fmaf(s16.y, c.x, ai); br = fmaf(d16.x, c.y, br); bi = fmaf(d16.y, c.y, bi); cr = fmaf(s16.x, e.x, cr); ci = fmaf(s16.y, e.x, ci); dr = fmaf(d16.x, e.y, dr); di = fmaf(d16.y, e.y, di); }
      { const float2 c = t[17], e = u[17]; ar = fmaf(s17.x, c.x, ar); ai = fmaf(s17.y, c.x, ai); br = fmaf(d17.x, c.y, br); bi = fmaf(d17.y, c.y, bi); cr = fmaf(s17.x, e.x, cr); ci = fmaf(s17.y, e.x, ci); dr = fmaf(d17.x, e.y, dr); di = fmaf(d17.y, e.y, di); }
      { const float2 c = t[18], e = u[18]; ar = fmaf(s18.x, c.x, ar); ai = fmaf(s18.y, c.x, ai); br = fmaf(d18.x, c.y, br); bi = fmaf(d18.y, c.y, bi); cr = fmaf(s18.x, e.x, cr); ci = fmaf(s18.y, e.x, ci); dr = fmaf(d18.x, e.y, dr); di = fmaf(d18.y, e.y, di); }
      { const float2 c = t[19], e = u[19]; ar = fmaf(s19.x, c.x, ar); ai = fmaf(s19.y, c.x, ai); br = fmaf(d19.x, c.y, br); bi = fmaf(d19.y, c.y, bi); cr = fmaf(s19.x, e.x, cr); ci = fmaf(s19.y, e.x, ci); dr = fmaf(d19.x, e.y, dr); di = fmaf(d19.y, e.y, di); }
      { const float2 c = t[20], e = u[20]; ar = fmaf(s20.x, c.x, ar); ai = fmaf(s20.y, c.x, ai); br = fmaf(d20.x, c.y, br); bi = fmaf(d20.y, c.y, bi); cr = fmaf(s20.x, e.x, cr); ci = fmaf(s20.y, e.x, ci); dr = fmaf(d20.x, e.y, dr); di = fmaf(d20.y, e.y, di); }
      { const float2 c = t[21], e = u[21]; ar = fmaf(s21.x, c.x, ar); ai = fmaf(s21.y, c.x, ai); br = fmaf(d21.x, c.y, br); bi = fmaf(d21.y, c.y, bi); cr = fmaf(s21.x, e.x, cr); ci = fmaf(s21.y, e.x, ci); dr = fmaf(d21.x, e.y, dr); di = fmaf(d21.y, e.y, di); }
      { const float2 c = t[22], e = u[22]; ar = fmaf(s22.x, c.x, ar); ai = fmaf(s22.y, c.x, ai); br = fmaf(d22.x, c.y, br); bi = fmaf(d22.y, c.y, bi); cr = fmaf(s22.x, e.x, cr); ci = fmaf(s22.y, e.x, ci); dr = fmaf(d22.x, e.y, dr); di = fmaf(d22.y, e.y, di); }
      { const float2 c = t[23], e = u[23]; ar = fmaf(s23.x, c.x, ar); ai = fmaf(s23.y, c.x, ai); br = fmaf(d23.x, c.y, br); bi = fmaf(d23.y, c.y, bi); cr = fmaf(s23.x, e.x, cr); ci = fmaf(s23.y, e.x, ci); dr = fmaf(d23.x, e.y, dr); di = fmaf(d23.y, e.y, di); }
      { const float2 c = t[24], e = u[24]; ar = fmaf(s24.x, c.x, ar); ai = fmaf(s24.y, c.x, ai); br = fmaf(d24.x, c.y, br); bi = fmaf(d24.y, c.y, bi); cr = fmaf(s24.x, e.x, cr); ci = fmaf(s24.y, e.x, ci); dr = fmaf(d24.x, e.y, dr); di = fmaf(d24.y, e.y, di); }
      { const float2 c = t[25], e = u[25]; ar = fmaf(s25.x, c.x, ar); ai = fmaf(s25.y, c.x, ai); br = fmaf(d25.x, c.y, br); bi = fmaf(d25.y, c.y, bi); cr = fmaf(s25.x, e.x, cr); ci = fmaf(s25.y, e.x, ci); dr = fmaf(d25.x, e.y, dr); di = fmaf(d25.y, e.y, di); }
      { const float2 c = t[26], e = u[26]; ar = fmaf(s26.x, c.x, ar); ai = fmaf(s26.y, c.x, ai); br = fmaf(d26.x, c.y, br); bi = fmaf(d26.y, c.y, bi); cr = fmaf(s26.x, e.x, cr); ci = fmaf(s26.y, e.x, ci); dr = fmaf(d26.x, e.y, dr); di = fmaf(d26.y, e.y, di); }
      const int k2 = k + 13;
      if (!INV) { st(k, make_float2(ar + bi, ai - br)); st(53 - k, make_float2(ar - bi, ai + br)); st(k2, make_float2(cr + di, ci - dr)); st(53 - k2, make_float2(cr - di, ci + dr)); }
      else { st(k, make_float2(ar - bi, ai + br)); st(53 - k, make_float2(ar + bi, ai - br)); st(k2, make_float2(cr - di, ci + dr)); st(53 - k2, make_float2(cr + di, ci - dr)); }
    }
  } else {
#pragma unroll 1
    for (int k = 1; k <= 26; k++) {
      const float2* t = c_tw53[k];
      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;
      { const float2 c = t[1]; ar = fmaf(s1.x, c.x, ar); ai = fmaf(s1.y, c.x, ai); br = fmaf(d1.x, c.y, br); bi = fmaf(d1.y, c.y, bi); }
      { const float2 c = t[2]; ar = fmaf(s2.x, c.x, ar); ai = fmaf(s2.y, c.x, ai); br = fmaf(d2.x, c.y, br); bi = fmaf(d2.y, c.y, bi); }
      { const float2 c = t[3]; ar = fmaf(s3.x, c.x, ar); ai = fmaf(s3.y, c.x, ai); br = fmaf(d3.x, c.y, br); bi = fmaf(d3.y, c.y, bi); }
      { const float2 c = t[4]; ar = fmaf(s4.x, c.x, ar); ai = fmaf(s4.y, c.x, ai); br = fmaf(d4.x, c.y, br); bi = fmaf(d4.y, c.y, bi); }
      { const float2 c = t[5]; ar = fmaf(s5.x, c.x, ar); ai = fmaf(s5.y, c.x, ai); br = fmaf(d5.x, c.y, br); bi = fmaf(d5.y, c.y, bi); }
      { const float2 c = t[6]; ar = fmaf(s6.x, c.x, ar); ai = fmaf(s6.y, c.x, ai); br = fmaf(d6.x, c.y, br); bi = fmaf(d6.y, c.y, bi); }
      { const float2 c = t[7]; ar = fmaf(s7.x, c.x, ar); ai = fmaf(s7.y, c.x, ai); br = fmaf(d7.x, c.y, br); bi = fmaf(d7.y, c.y, bi); }
      { const float2 c = t[8]; ar = fmaf(s8.x, c.x, ar); ai = fmaf(s8.y, c.x, ai); br = fmaf(d8.x, c.y, br); bi = fmaf(d8.y, c.y, bi); }
      { const float2 c = t[9]; ar = fmaf(s9.x, c.x, ar); ai = fmaf(s9.y, c.x, ai); br = fmaf(d9.x, c.y, br); bi = fmaf(d9.y, c.y, bi); }
      { const float2 c = t[10]; ar = fmaf(s10.x, c.x, ar); ai = fmaf(s10.y, c.x, ai); br = fmaf(d10.x, c.y, br); bi = fmaf(d10.y, c.y, bi); }
      { const float2 c = t[11]; ar = fmaf(s11.x, c.x, ar); ai = fmaf(s11.y, c.x, ai); br = fmaf(d11.x, c.y, br); bi = fmaf(d11.y, c.y, bi); }
      { const float2 c = t[12]; ar = fmaf(s12.x, c.x, ar); ai = fmaf(s12.y, c.x, ai); br = fmaf(d12.x, c.y, br); bi = fmaf(d12.y, c.y, bi); }
      { const float2 c = t[13]; ar = fmaf(s13.x, c.x, ar); ai = fmaf(s13.y, c.x, ai); br = fmaf(d13.x, c.y, br); bi = fmaf(d13.y, c.y, bi); }
      { const float2 c = t[14]; ar = fmaf(s14.x, c.x, ar); ai = fmaf(s14.y, c.x, ai); br = fmaf(d14.x, c.y, br); bi = fmaf(d14.y, c.y, bi); }
      { const float2 c = t[15]; ar = fmaf(s15.x, c.x, ar); ai = fmaf(s15.y, c.x, ai); br = fmaf(d15.x, c.y, br); bi = fmaf(d15.y, c.y, bi); }
      { const float2 c = t[16]; ar = fmaf(s16.x, c.x, ar); ai = fmaf(s16.y, c.x, ai); br = fmaf(d16.x, c.y, br); bi = fmaf(d16.y, c.y, bi); }
      { const float2 c = t[17]; ar = fmaf(s17.x, c.x, ar); ai = fmaf(s17.y, c.x, ai); br = fmaf(d17.x, c.y, br); bi = fmaf(d17.y, c.y, bi); }
      { const float2 c = t[18]; ar = fmaf(s18.x, c.x, ar); ai = fmaf(s18.y, c.x, ai); br = fmaf(d18.x, c.y, br); bi = fmaf(d18.y, c.y, bi); }
      { const float2 c = t[19]; ar = fmaf(s19.x, c.x, ar); ai = fmaf(s19.y, c.x, ai); br = fmaf(d19.x, c.y, br); bi = fmaf(d19.y, c.y, bi); }
      { const float2 c = t[20]; ar = fmaf(s20.x, c.x, ar); ai = fmaf(s20.y, c.x, ai); br = fmaf(d20.x, c.y, br); bi = fmaf(d20.y, c.y, bi); }
      { const float2 c = t[21]; ar = fmaf(s21.x, c.x, ar); ai = fmaf(s21.y, c.x, ai); br = fmaf(d21.x, c.y, br); bi = fmaf(d21.y, c.y, bi); }
      { const float2 c = t[22]; ar = fmaf(s22.x, c.x, ar); ai = fmaf(s22.y, c.x, ai); br = fmaf(d22.x, c.y, br); bi = fmaf(d22.y, c.y, bi); }
      { const float2 c = t[23]; ar = fmaf(s23.x, c.x, ar); ai = fmaf(s23.y, c.x, ai); br = fmaf(d23.x, c.y, br); bi = fmaf(d23.y, c.y, bi); }
      { const float2 c = t[24]; ar = fmaf(s24.x, c.x, ar); ai = fmaf(s24.y, c.x, ai); br = fmaf(d24.x, c.y, br); bi = fmaf(d24.y, c.y, bi); }
      { const float2 c = t[25]; ar = fmaf(s25.x, c.x, ar); ai = fmaf(s25.y, c.x, ai); br = fmaf(d25.x, c.y, br); bi = fmaf(d25.y, c.y, bi); }
      { const float2 c = t[26]; ar = fmaf(s26.x, c.x, ar); ai = fmaf(s26.y, c.x, ai); br = fmaf(d26.x, c.y, br); bi = fmaf(d26.y, c.y, bi); }
      if (!INV) { st(k, make_float2(ar + bi, ai - br)); st(53 - (k), make_float2(ar - bi, ai + br)); }
      else { st(k, make_float2(ar - bi, ai + br)); st(53 - (k), make_float2(ar + bi, ai - br)); }
    }
  }
}
}  // namespace mc
