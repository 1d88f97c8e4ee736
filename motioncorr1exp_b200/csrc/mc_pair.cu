// Pair stage of libmc (sm_100a): cross power x B-factor with the inverse
// along ky pruned to the pbx rows (cufunc.cu:343-370), and the pruned C2R
// along kx onto the pbx window (cufunc.cu:229-233, 404-407).
#include <algorithm>

// The column stage's Q-point codelets use packed FP32 FMAs in their odd-radix
// butterflies (bitwise the scalar results; 3 % faster here, while the
// forward kernels' 70-point codelets spill more with them).
#define MC_PACKED_FMA 1
#include "kcommon.cuh"

namespace mc {

// ============================================================ pair columns ==
size_t pair_cols_smem(int n, int P, int Q, int box) {
  const size_t outer = pair_cols_tabn(n, P, box) ? (size_t)n : (size_t)P * box;
  return (size_t)2 * n * sizeof(float2)     // ping-pong
         + (size_t)n * sizeof(float)        // B-factor column
         + (size_t)Q * sizeof(float2)       // inner twiddles
         + outer * sizeof(float2);          // outer twiddles
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
  const bool tabn = a.twN != nullptr;
  copy_table(twQ, a.twQ, Q);
  if (tabn) copy_table(twO, a.twN, n);
  else copy_table(twO, a.twO, P * box);
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
        if (tabn) {
          const int y = (a.ystart + m) % n;
          int e = (int)(((long long)k0 * y) % n);
          for (int k = k0; k < k1; k++) {
            const float2 t = twO[e];
            const float2 yv = yr[k];
            acc.x = fmaf(t.x, yv.x, fmaf(-t.y, yv.y, acc.x));
            acc.y = fmaf(t.x, yv.y, fmaf(t.y, yv.x, acc.y));
            e += y;
            if (e >= n) e -= n;
          }
        } else {
          for (int k = k0; k < k1; k++) {
            const float2 t = twO[k * box + m];
            const float2 yv = yr[k];
            acc.x = fmaf(t.x, yv.x, fmaf(-t.y, yv.y, acc.x));
            acc.y = fmaf(t.x, yv.y, fmaf(t.y, yv.x, acc.y));
          }
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
      fft_reg_pf<Q, true>(x);
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

// ---- split n = P x Q fixed at compile time ----------------------------------
// The gather reads the stride-P subsequence at immediate offsets.  The outer
// sum out[m] = sum_k1 Y[r(m)][k1] W^(k1 y_m), r(m) = (ystart + m) mod Q, runs
// as items (output row m, chunk of at most 16 k1): Horner's rule from the
// chunk's last term down, acc = acc w + Y with w = W^(y_m) (4 FMAs per term,
// no twiddle loads; the powers of the rounded w drift by ~1e-6 over a chunk),
// then one multiply by W^(kb y_m).  A thread runs three items at a time with
// their chains interleaved (one item 5.85, two 5.71, three 5.64 ms per c2
// movie: with two warps per scheduler the dependent FMAs of one item left
// issue slots empty).  Consecutive threads take consecutive rows
// m, so their Y rows (odd stride in float2) fall on different bank pairs and
// their twiddle loads are contiguous.  The chunk partials meet in shared
// memory and are added in chunk order.
template <int Q, int P>
struct RpShape {
  static constexpr int T = P <= 32 ? 32 : (P <= 64 ? 64 : 128);  // team threads
  static constexpr int W = T / 32;                                // chunk count granule
  static constexpr int C = ((P + 15) / 16 + W - 1) / W * W;       // k1 chunks (96 C / T whole)
  static constexpr int L = (P + C - 1) / C;                       // chunk length <= 16
  static constexpr int PS = P | 1;                                // odd Y row stride (float2)
  static constexpr int YN = Q * PS;
};

size_t pair_cols_rp_smem(int n, int yn, int team, int chunks, int box) {
  const int teams = kRegThreads / team;
  return (size_t)((n + 1) / 2) * sizeof(float2) + (size_t)(chunks + 1) * box * sizeof(float2) +
         (size_t)teams * ((size_t)yn + (size_t)chunks * box) * sizeof(float2);
}

template <int Q, int P>
__global__ void __launch_bounds__(kRegThreads, pair_reg_min_blocks(Q)) k_pair_cols_rp(PairColsArgs a) {
  using S = RpShape<Q, P>;
  constexpr int T = S::T, C = S::C, L = S::L, N = P * Q, PS = S::PS, YN = S::YN;
  extern __shared__ float2 sm[];
  const int box = a.box;
  float* wcol = reinterpret_cast<float*>(sm);
  // twiddle rows the sums need: tws[0][m] = W^(y_m) (twO row 1), tws[1 + c][m]
  // = W^(kb(c) y_m) (twO row c L)
  float2* tws = sm + (N + 1) / 2;
  constexpr int teams = kRegThreads / T;
  const int tid = threadIdx.x;
  const int tm = tid / T, lt = tid - tm * T;
  float2* Y = tws + (C + 1) * box + (size_t)tm * (YN + C * box);
  float2* part = Y + YN;
  const int kx = blockIdx.y;
  for (int ky = tid; ky < N; ky += kRegThreads) {
    const int y = ky < N / 2 ? ky : ky - N;
    wcol[ky] = expf(a.mbf * (float)(kx * kx + y * y)) * a.inv_size;
  }
  for (int i = tid; i < (C + 1) * box; i += kRegThreads) {
    const int row = i / box, m = i - row * box;
    const int k = row == 0 ? 1 : min((row - 1) * L, P - 1);
    tws[i] = __ldg(a.twO + (long long)k * box + m);
  }
  __syncthreads();
  const int ys = a.ystart % Q;
  const int p0 = blockIdx.x * a.pairs_per_cta;
  const int p1 = min(p0 + a.pairs_per_cta, a.npairs);
  for (int p = p0 + tm; p < p1; p += teams) {
    const int2 pr = a.pairs[p];
    if (lt < P) {
      const float2* ca = a.specA + (long long)pr.x * a.strideA + (long long)kx * a.ldn + lt;
      const float2* cb = a.specB + (long long)pr.y * a.strideB + (long long)kx * a.ldn + lt;
      const float* wc = wcol + lt;
      float2 x[Q];
#pragma unroll
      for (int k2 = 0; k2 < Q; k2++) x[k2] = cscale(cmulc(__ldg(ca + P * k2), __ldg(cb + P * k2)), wc[P * k2]);
      fft_reg_pf<Q, true>(x);
#pragma unroll
      for (int r = 0; r < Q; r++) Y[lt + PS * r] = x[r];
    }
    team_barrier(1 + tm, T);
    int c = lt / box, m = lt - (lt / box) * box;
    // three items per pass, their chains interleaved (three times the
    // independent work)
    for (int it = lt; it < box * C; it += 3 * T) {
      int c1 = c, m1 = m + T;
      while (m1 >= box) {
        m1 -= box;
        c1++;
      }
      int c2 = c1, m2 = m1 + T;
      while (m2 >= box) {
        m2 -= box;
        c2++;
      }
      const bool has1 = it + T < box * C, has2 = it + 2 * T < box * C;
      const int nc_ = c2, nm_ = m2;
      if (!has1) {
        c1 = c;
        m1 = m;
      }
      if (!has2) {
        c2 = c;
        m2 = m;
      }
      int r0 = ys + m % Q, r1 = ys + m1 % Q, r2 = ys + m2 % Q;
      if (r0 >= Q) r0 -= Q;
      if (r1 >= Q) r1 -= Q;
      if (r2 >= Q) r2 -= Q;
      const int kb0 = c * L, kb1 = c1 * L, kb2 = c2 * L;
      const float2* yr0 = Y + PS * r0 + kb0;
      const float2* yr1 = Y + PS * r1 + kb1;
      const float2* yr2 = Y + PS * r2 + kb2;
      const float2 w0 = tws[m], w1 = tws[m1], w2 = tws[m2];
      const float2 v0 = cmul(w0, w0), v1 = cmul(w1, w1), v2 = cmul(w2, w2);
      float2 ae0 = make_float2(0.f, 0.f), ao0 = make_float2(0.f, 0.f);
      float2 ae1 = make_float2(0.f, 0.f), ao1 = make_float2(0.f, 0.f);
      float2 ae2 = make_float2(0.f, 0.f), ao2 = make_float2(0.f, 0.f);
#pragma unroll
      for (int kk = L - 1; kk >= 0; kk--) {
        if (L * C == P || kb0 + kk < P) {
          const float2 yv = yr0[kk];
          float2& h = (kk & 1) ? ao0 : ae0;
          const float2 s = h;
          h.x = fmaf(s.x, v0.x, fmaf(-s.y, v0.y, yv.x));
          h.y = fmaf(s.x, v0.y, fmaf(s.y, v0.x, yv.y));
        }
        if (L * C == P || kb1 + kk < P) {
          const float2 yv = yr1[kk];
          float2& h = (kk & 1) ? ao1 : ae1;
          const float2 s = h;
          h.x = fmaf(s.x, v1.x, fmaf(-s.y, v1.y, yv.x));
          h.y = fmaf(s.x, v1.y, fmaf(s.y, v1.x, yv.y));
        }
        if (L * C == P || kb2 + kk < P) {
          const float2 yv = yr2[kk];
          float2& h = (kk & 1) ? ao2 : ae2;
          const float2 s = h;
          h.x = fmaf(s.x, v2.x, fmaf(-s.y, v2.y, yv.x));
          h.y = fmaf(s.x, v2.y, fmaf(s.y, v2.x, yv.y));
        }
      }
      float2 acc0, acc1, acc2;
      acc0.x = fmaf(ao0.x, w0.x, fmaf(-ao0.y, w0.y, ae0.x));
      acc0.y = fmaf(ao0.x, w0.y, fmaf(ao0.y, w0.x, ae0.y));
      acc1.x = fmaf(ao1.x, w1.x, fmaf(-ao1.y, w1.y, ae1.x));
      acc1.y = fmaf(ao1.x, w1.y, fmaf(ao1.y, w1.x, ae1.y));
      acc2.x = fmaf(ao2.x, w2.x, fmaf(-ao2.y, w2.y, ae2.x));
      acc2.y = fmaf(ao2.x, w2.y, fmaf(ao2.y, w2.x, ae2.y));
      if (kb0 < P) acc0 = cmul(acc0, tws[(1 + c) * box + m]);
      if (kb1 < P) acc1 = cmul(acc1, tws[(1 + c1) * box + m1]);
      if (kb2 < P) acc2 = cmul(acc2, tws[(1 + c2) * box + m2]);
      part[c * box + m] = acc0;
      if (has1) part[c1 * box + m1] = acc1;
      if (has2) part[c2 * box + m2] = acc2;
      m = nm_ + T;
      c = nc_;
      while (m >= box) {
        m -= box;
        c++;
      }
    }
    team_barrier(1 + tm, T);
    for (int m = lt; m < box; m += T) {
      float2 s = part[m];
#pragma unroll
      for (int c = 1; c < C; c++) s = cadd(s, part[c * box + m]);
      a.G[((long long)p * a.H + kx) * box + m] = s;
    }
    // the next pair writes Y before its first barrier and part after it:
    // every read of this pair's Y precedes the second barrier above, and every
    // read of part precedes the next pair's first barrier
  }
}

// ---- row stage with the same compiled split --------------------------------
// box[p][yb][xb] = sum_kx h(kx) Re(G[p][kx][yb] exp(+2 pi i kx x_xb / n)) is
// the length-n inverse DFT of the Hermitian extension of row yb (real parts
// at kx = 0 and n/2, conj(G[n - kx]) above n/2), evaluated at the box's
// columns.  Two rows ride in one complex sequence z = Ga + i Gb, so the real
// and imaginary parts of the result are the two output rows.  A CTA stages
// G[p][:, 2 teams rows] (coalesced, odd row stride), each team gathers its
// row pair, runs the inverse Q-point codelet on the stride-P subsequences and
// forms the box columns by the column stage's Horner sums.
template <int Q, int P>
__host__ __device__ __forceinline__ size_t pair_rows_rp_region(int H) {
  using S = RpShape<Q, P>;
  constexpr int teams = kRegThreads / S::T;
  const size_t g = (size_t)H * (2 * teams + 1);
  const size_t y = (size_t)teams * S::YN;
  return g > y ? g : y;
}

template <int Q, int P>
size_t pair_rows_rp_smem(int H, int box) {
  using S = RpShape<Q, P>;
  constexpr int teams = kRegThreads / S::T;
  return (pair_rows_rp_region<Q, P>(H) + (size_t)(S::C + 1) * box + (size_t)teams * S::C * box) * sizeof(float2);
}

template <int Q, int P>
__global__ void __launch_bounds__(kRegThreads, pair_reg_min_blocks(Q)) k_pair_rows_rp(PairRowsArgs a, const float2* __restrict__ twO,
                                                                                        int ystart) {
  using S = RpShape<Q, P>;
  constexpr int T = S::T, C = S::C, L = S::L, N = P * Q, PS = S::PS;
  constexpr int teams = kRegThreads / T, R = 2 * teams, RS = R + 1;
  extern __shared__ float2 sm[];
  const int box = a.box, H = a.H;
  float2* reg = sm;                                    // staged G rows, then the teams' Y
  float2* tws = sm + pair_rows_rp_region<Q, P>(H);
  float2* part0 = tws + (C + 1) * box;
  const int tid = threadIdx.x, tm = tid / T, lt = tid - tm * T;
  const int p = blockIdx.x, yb0 = blockIdx.y * R;
  const float2* G = a.G + (long long)p * H * box;
  for (int i = tid; i < H * R; i += kRegThreads) {
    const int kx = i / R, r = i - kx * R;
    reg[kx * RS + r] = yb0 + r < box ? G[(long long)kx * box + yb0 + r] : make_float2(0.f, 0.f);
  }
  for (int i = tid; i < (C + 1) * box; i += kRegThreads) {
    const int row = i / box, m = i - row * box;
    const int k = row == 0 ? 1 : min((row - 1) * L, P - 1);
    tws[i] = __ldg(twO + (long long)k * box + m);
  }
  __syncthreads();
  float2 x[Q];
  if (lt < P) {
    const int ra = 2 * tm, rb = ra + 1;
#pragma unroll
    for (int k2 = 0; k2 < Q; k2++) {
      const int kx = lt + P * k2;
      float2 z;
      if (kx == 0 || 2 * kx == N) {
        z = make_float2(reg[kx * RS + ra].x, reg[kx * RS + rb].x);
      } else if (2 * kx < N) {
        const float2 ga = reg[kx * RS + ra], gb = reg[kx * RS + rb];
        z = make_float2(ga.x - gb.y, ga.y + gb.x);
      } else {
        const int kr = N - kx;
        const float2 ga = reg[kr * RS + ra], gb = reg[kr * RS + rb];
        z = make_float2(ga.x + gb.y, gb.x - ga.y);
      }
      x[k2] = z;
    }
    fft_reg_pf<Q, true>(x);
  }
  __syncthreads();  // every team has gathered: the staged rows give way to Y
  float2* Y = reg + (size_t)tm * S::YN;
  float2* part = part0 + (size_t)tm * C * box;
  if (lt < P) {
#pragma unroll
    for (int r = 0; r < Q; r++) Y[lt + PS * r] = x[r];
  }
  team_barrier(1 + tm, T);
  const int ys = ystart % Q;
  int c = lt / box, m = lt - (lt / box) * box;
  for (int it = lt; it < box * C; it += T) {
    int r = ys + m % Q;
    if (r >= Q) r -= Q;
    const int kb = c * L;
    const float2* yr = Y + PS * r + kb;
    const float2 w = tws[m];
    const float2 w2 = cmul(w, w);
    float2 ae = make_float2(0.f, 0.f), ao = make_float2(0.f, 0.f);
#pragma unroll
    for (int kk = L - 1; kk >= 0; kk--) {
      if (L * C == P || kb + kk < P) {
        const float2 yv = yr[kk];
        float2& h = (kk & 1) ? ao : ae;
        const float2 s = h;
        h.x = fmaf(s.x, w2.x, fmaf(-s.y, w2.y, yv.x));
        h.y = fmaf(s.x, w2.y, fmaf(s.y, w2.x, yv.y));
      }
    }
    float2 acc;
    acc.x = fmaf(ao.x, w.x, fmaf(-ao.y, w.y, ae.x));
    acc.y = fmaf(ao.x, w.y, fmaf(ao.y, w.x, ae.y));
    if (kb < P) acc = cmul(acc, tws[(1 + c) * box + m]);
    else acc = make_float2(0.f, 0.f);
    part[c * box + m] = acc;
    m += T;
    while (m >= box) {
      m -= box;
      c++;
    }
  }
  team_barrier(1 + tm, T);
  const int ya = yb0 + 2 * tm, yb = ya + 1;
  for (int mm = lt; mm < box; mm += T) {
    float2 s = part[mm];
#pragma unroll
    for (int cc = 1; cc < C; cc++) s = cadd(s, part[cc * box + mm]);
    if (ya < box) a.boxes[((long long)p * box + ya) * box + mm] = s.x;
    if (yb < box) a.boxes[((long long)p * box + yb) * box + mm] = s.y;
  }
}

// the compiled (Q, P) splits of the tuned lengths: 3710, 4096, 2048, 1024
#define MC_RP_LIST(X) X(35, 106) X(70, 53) X(64, 64) X(32, 128) X(64, 32) X(32, 64) X(16, 128) X(32, 32) X(16, 64)

bool pair_cols_rp_supported(int P, int Q) {
#define MC_RP_HAS(A, B) if (Q == (A) && P == (B)) return true;
  MC_RP_LIST(MC_RP_HAS)
#undef MC_RP_HAS
  return false;
}

size_t pair_cols_launch_smem(int n, int P, int Q, int box) {
#define MC_RP_SMEM(A, B) \
  if (Q == (A) && P == (B)) return pair_cols_rp_smem(n, RpShape<A, B>::YN, RpShape<A, B>::T, RpShape<A, B>::C, box);
  MC_RP_LIST(MC_RP_SMEM)
#undef MC_RP_SMEM
  if (pair_cols_reg_supported(P, Q)) return pair_cols_reg_smem(n, P <= 32 ? 32 : (P <= 64 ? 64 : 128));
  return pair_cols_smem(n, P, Q, box) + 16;
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
#define MC_RP_LAUNCH(A, B)                                                                                  \
  if (a.Q == (A) && a.P == (B) && a.n == (A) * (B)) {                                                      \
    const size_t smem = pair_cols_rp_smem(a.n, RpShape<A, B>::YN, RpShape<A, B>::T, RpShape<A, B>::C, a.box); \
    cudaError_t e = allow_smem((const void*)k_pair_cols_rp<A, B>, smem);                                   \
    if (e != cudaSuccess) return e;                                                                        \
    k_pair_cols_rp<A, B><<<grid, kRegThreads, smem, st>>>(a);                                              \
    return cudaGetLastError();                                                                             \
  }
  MC_RP_LIST(MC_RP_LAUNCH)
#undef MC_RP_LAUNCH
  if (pair_cols_reg_supported(a.P, a.Q)) {
    const int team = a.P <= 32 ? 32 : (a.P <= 64 ? 64 : 128);
    return dispatch_reg(a, team, pair_cols_reg_smem(a.n, team), grid, st);
  }
  // the shared-memory size assumes the outer table the kernel will copy
  if ((a.twN != nullptr) != pair_cols_tabn(a.n, a.P, a.box)) return cudaErrorInvalidValue;
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
  if (a.twO) {
#define MC_RP_ROWS(A, B)                                                                            \
  if (a.Q == (A) && a.P == (B) && 2 * (a.H - 1) == (A) * (B)) {                                    \
    constexpr int rows = 2 * (kRegThreads / RpShape<A, B>::T);                                     \
    const size_t smem = pair_rows_rp_smem<A, B>(a.H, a.box);                                       \
    if (smem > 227 * 1024) return cudaErrorInvalidValue;                                            \
    cudaError_t e = allow_smem((const void*)k_pair_rows_rp<A, B>, smem);                           \
    if (e != cudaSuccess) return e;                                                                 \
    k_pair_rows_rp<A, B><<<dim3(a.npairs, (a.box + rows - 1) / rows), kRegThreads, smem, st>>>(a, a.twO, a.ystart); \
    return cudaGetLastError();                                                                      \
  }
    MC_RP_LIST(MC_RP_ROWS)
#undef MC_RP_ROWS
  }
  k_pair_rows<<<a.npairs, kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mc
