// Device-side FP64 drift solve (single CTA): the same computation as the host
// lsq.cpp path (DFAlign.cu:914-948, mfunc.h:86-146), so a whole movie can run
// on the plan stream without a host round trip (and be captured in a graph).
//
//   1. s = argmin |A s - b| over all rows (normal equations, Cholesky)
//   2. ki1 = |A s - b|; rows ranked by ascending ki1 (ties: lower row first)
//   3. keep the prefix ending at the last rank >= ncol with ki1 < kithresh
//      (else the first ncol rows), then add rows in rank order until the pair
//      graph is connected (rank(A) = nframe - components)
//   4. s = argmin over the kept rows; ki2 over the kept rows
//   5. per-step shifts, cumulative frame shifts and the sum shifts
//      s_k = -total_k + mid of DFAlign.cu:1114-1181 for the summed frames
#include <math.h>

#include "kernels.cuh"

namespace mc {

namespace {

constexpr int kSolveThreads = 256;

__device__ int uf_find(int* par, int x) {
  while (par[x] != x) {
    par[x] = par[par[x]];
    x = par[x];
  }
  return x;
}

// Normal equations over the masked rows, Cholesky, two substitutions.
// Returns false (in every thread) when a pivot is not positive.
__device__ bool solve_masked(const SolveArgs& a, const int* mask, double* sx, double* sy) {
  const int P = a.npairs, nc = a.nframe - 1, tid = threadIdx.x;
  double* M = a.M;
  double* rx = a.rhs;
  double* ry = a.rhs + nc;
  __shared__ int s_bad;
  if (tid == 0) s_bad = 0;
  for (int idx = tid; idx < nc * nc; idx += kSolveThreads) {
    const int k = idx / nc, l = idx - (idx / nc) * nc;
    const int lo = min(k, l), hi = max(k, l);
    int cnt = 0;
    for (int r = 0; r < P; r++)
      if (mask[r] && a.pairs[r].x <= lo && hi < a.pairs[r].y) cnt++;
    M[idx] = (double)cnt;
  }
  for (int k = tid; k < nc; k += kSolveThreads) {
    double x = 0.0, y = 0.0;
    for (int r = 0; r < P; r++)
      if (mask[r] && a.pairs[r].x <= k && k < a.pairs[r].y) {
        x += (double)a.pshift[2 * r];
        y += (double)a.pshift[2 * r + 1];
      }
    rx[k] = x;
    ry[k] = y;
  }
  __syncthreads();
  double dmax = 1.0;
  for (int k = 0; k < nc; k++) dmax = fmax(dmax, M[k * nc + k]);
  const double tiny = 1e-12 * dmax;
  for (int k = 0; k < nc; k++) {
    if (tid == 0) {
      const double d = M[k * nc + k];
      if (!(d > tiny)) s_bad = 1;
      M[k * nc + k] = sqrt(fmax(d, tiny));
    }
    __syncthreads();
    const double lkk = M[k * nc + k];
    for (int i = k + 1 + tid; i < nc; i += kSolveThreads) M[i * nc + k] /= lkk;
    __syncthreads();
    const int m = nc - k - 1;
    for (int idx = tid; idx < m * m; idx += kSolveThreads) {
      const int i = k + 1 + idx / m, j = k + 1 + idx % m;
      if (j <= i) M[i * nc + j] -= M[i * nc + k] * M[j * nc + k];
    }
    __syncthreads();
  }
  if (tid == 0) {
    for (int i = 0; i < nc; i++) {
      double vx = rx[i], vy = ry[i];
      for (int m2 = 0; m2 < i; m2++) {
        vx -= M[i * nc + m2] * rx[m2];
        vy -= M[i * nc + m2] * ry[m2];
      }
      rx[i] = vx / M[i * nc + i];
      ry[i] = vy / M[i * nc + i];
    }
    for (int i = nc - 1; i >= 0; i--) {
      double vx = rx[i], vy = ry[i];
      for (int m2 = i + 1; m2 < nc; m2++) {
        vx -= M[m2 * nc + i] * sx[m2];
        vy -= M[m2 * nc + i] * sy[m2];
      }
      sx[i] = vx / M[i * nc + i];
      sy[i] = vy / M[i * nc + i];
    }
  }
  __syncthreads();
  return s_bad == 0;
}

}  // namespace

__global__ void __launch_bounds__(kSolveThreads) k_solve(SolveArgs a) {
  const int P = a.npairs, nf = a.nframe, nc = nf - 1, tid = threadIdx.x;
  double* sx = a.shift;       // [nc][2] interleaved at the end; work arrays first
  double* wx = a.work;        // [nc]
  double* wy = a.work + nc;   // [nc]
  double* cx = a.work + 2 * nc;  // prefix sums [nf]
  double* cy = a.work + 2 * nc + nf;
  int* mask = a.mask;
  int* order = a.order;
  for (int r = tid; r < P; r += kSolveThreads) mask[r] = 1;
  __syncthreads();
  if (!solve_masked(a, mask, wx, wy)) {
    if (tid == 0) *a.status = -6;
    return;
  }
  // residuals of the first solve via prefix sums of the steps
  if (tid == 0) {
    cx[0] = cy[0] = 0.0;
    for (int k = 0; k < nc; k++) {
      cx[k + 1] = cx[k] + wx[k];
      cy[k + 1] = cy[k] + wy[k];
    }
  }
  __syncthreads();
  for (int r = tid; r < P; r += kSolveThreads) {
    const int i = a.pairs[r].x, j = a.pairs[r].y;
    // sum of the steps in [i, j) accumulated like the host (k ascending)
    double ax = 0.0, ay = 0.0;
    for (int k = i; k < j; k++) {
      ax += wx[k];
      ay += wy[k];
    }
    const double dx = ax - (double)a.pshift[2 * r], dy = ay - (double)a.pshift[2 * r + 1];
    a.ki1[r] = sqrt(dx * dx + dy * dy);
  }
  __syncthreads();
  // stable ascending rank of ki1 (OD_Threshold's repeated first-minimum pick)
  for (int r = tid; r < P; r += kSolveThreads) {
    const double v = a.ki1[r];
    int pos = 0;
    for (int q = 0; q < P; q++) {
      const double u = a.ki1[q];
      pos += (u < v || (u == v && q < r)) ? 1 : 0;
    }
    order[pos] = r;
  }
  __syncthreads();
  if (tid == 0) {
    int i;
    for (i = P - 1; i >= nc; i--)
      if (a.ki1[order[i]] < (double)a.kithresh) break;
    int len = i + 1;
    int* par = a.uf;
    for (int f = 0; f < nf; f++) par[f] = f;
    int comps = nf;
    for (int q = 0; q < P; q++) mask[q] = 0;
    auto add = [&](int row) {
      mask[row] = 1;
      const int x = uf_find(par, a.pairs[row].x), y = uf_find(par, a.pairs[row].y);
      if (x != y) {
        par[x] = y;
        comps--;
      }
    };
    for (int q = 0; q < len && q < P; q++) add(order[q]);
    while (comps > 1 && len < P) add(order[len++]);
    *a.nkept = min(len, P);
  }
  __syncthreads();
  if (!solve_masked(a, mask, wx, wy)) {
    if (tid == 0) *a.status = -6;
    return;
  }
  if (tid == 0) {
    // kept rows in ascending order with their second-round residuals
    int q = 0;
    for (int r = 0; r < P; r++) {
      if (!mask[r]) continue;
      double ax = 0.0, ay = 0.0;
      for (int k = a.pairs[r].x; k < a.pairs[r].y; k++) {
        ax += wx[k];
        ay += wy[k];
      }
      const double dx = ax - (double)a.pshift[2 * r], dy = ay - (double)a.pshift[2 * r + 1];
      a.kept[q] = r;
      a.ki2[q] = sqrt(dx * dx + dy * dy);
      q++;
    }
    // steps -> oldshift -> steps (DFAlign.cu:958-962, 1061-1071), cumulative shifts
    double ox = 0.0, oy = 0.0, px = 0.0, py = 0.0, tx = 0.0, ty = 0.0;
    a.frame_shift[0] = 0.0;
    a.frame_shift[1] = 0.0;
    for (int k = 0; k < nc; k++) {
      const double nx = ox + wx[k], ny = oy + wy[k];  // newshift[k+1] = allshift + shift[k]
      ox = nx;
      oy = ny;
      const double stx = nx - px, sty = ny - py;     // oldshift[k+1] - oldshift[k]
      px = nx;
      py = ny;
      sx[2 * k] = stx;
      sx[2 * k + 1] = sty;
      tx += stx;
      ty += sty;
      a.frame_shift[2 * (k + 1)] = tx;
      a.frame_shift[2 * (k + 1) + 1] = ty;
    }
    // sum shifts (DFAlign.cu:1114-1181)
    double mx = 0.0, my = 0.0;
    if (a.align_to_mid)
      for (int k = 0; k < a.mid_steps; k++) {
        mx += sx[2 * k];
        my += sx[2 * k + 1];
      }
    double Tx = 0.0, Ty = 0.0;
    for (int k = 1; k < a.sum_first + 1; k++) {
      Tx += sx[2 * (k - 1)];
      Ty += sx[2 * (k - 1) + 1];
    }
    for (int k = a.sum_first; k <= a.sum_last; k++) {
      if (k > a.sum_first) {
        Tx += sx[2 * (k - 1)];
        Ty += sx[2 * (k - 1) + 1];
      }
      const int q2 = k - a.sum_first;
      a.sum_shift[q2] = make_double2(-Tx + mx, -Ty + my);
      a.sum_frames[q2] = k;
      a.sum_apply[q2] = (k == a.sum_first && !a.align_to_mid) ? 0 : 1;
    }
    *a.status = 0;
  }
}

// ---------------------------------------------------------------------------
// Shared-memory form of the same solve (used when its working set fits):
// the pair list, the measured shifts, the normal matrix, the residuals, the
// rank order, the union-find parents and the final step shifts live in
// shared memory (the one-thread sections, the threshold scan and the
// union-find pass, then run on shared-memory latency instead of dependent
// global loads); the normal equations are built one frame step per thread in
// a single pass over the pairs (a histogram of the pair ends per step, then
// suffix sums), and the per-row residual and compaction loops run in
// parallel.  Sums run in the same order as the global-memory form.
namespace {

struct SolveSmem {
  int2* pr;        // [P]
  float2* ps;      // [P]
  int* mask;       // [P]
  double* ki;      // [P]
  int* hist;       // [nc][nf]
  int* order;      // [P] rows in ascending ki1 rank
  int* uf;         // [nf] union-find parents
  double* M;       // [nc][nc]
  double* rx;      // [nc]
  double* ry;      // [nc]
};

__device__ bool solve_masked_smem(const SolveSmem& m, int P, int nf, double* sx, double* sy) {
  const int nc = nf - 1, tid = threadIdx.x;
  __shared__ int s_bad;
  if (tid == 0) s_bad = 0;
  // step k: rows with i <= k < j; histogram of their ends j and rhs sums
  for (int k = tid; k < nc; k += kSolveThreads) {
    int* h = m.hist + (size_t)k * nf;
    for (int j = 0; j < nf; j++) h[j] = 0;
    double x = 0.0, y = 0.0;
    for (int r = 0; r < P; r++) {
      const int2 q = m.pr[r];
      if (m.mask[r] && q.x <= k && k < q.y) {
        h[q.y]++;
        x += (double)m.ps[r].x;
        y += (double)m.ps[r].y;
      }
    }
    m.rx[k] = x;
    m.ry[k] = y;
    // M[k][l] (l >= k) = rows with i <= k and j > l: suffix sums of the ends
    int c = 0;
    for (int l = nc - 1; l >= k; l--) {
      c += h[l + 1];
      m.M[(size_t)k * nc + l] = (double)c;
      m.M[(size_t)l * nc + k] = (double)c;
    }
  }
  __syncthreads();
  double dmax = 1.0;
  for (int k = 0; k < nc; k++) dmax = fmax(dmax, m.M[(size_t)k * nc + k]);
  const double tiny = 1e-12 * dmax;
  double* M = m.M;
  for (int k = 0; k < nc; k++) {
    if (tid == 0) {
      const double d = M[(size_t)k * nc + k];
      if (!(d > tiny)) s_bad = 1;
      M[(size_t)k * nc + k] = sqrt(fmax(d, tiny));
    }
    __syncthreads();
    const double lkk = M[(size_t)k * nc + k];
    for (int i = k + 1 + tid; i < nc; i += kSolveThreads) M[(size_t)i * nc + k] /= lkk;
    __syncthreads();
    const int w = nc - k - 1;
    for (int idx = tid; idx < w * w; idx += kSolveThreads) {
      const int i = k + 1 + idx / w, j = k + 1 + idx % w;
      if (j <= i) M[(size_t)i * nc + j] -= M[(size_t)i * nc + k] * M[(size_t)j * nc + k];
    }
    __syncthreads();
  }
  if (tid == 0) {
    for (int i = 0; i < nc; i++) {
      double vx = m.rx[i], vy = m.ry[i];
      for (int q = 0; q < i; q++) {
        vx -= M[(size_t)i * nc + q] * m.rx[q];
        vy -= M[(size_t)i * nc + q] * m.ry[q];
      }
      m.rx[i] = vx / M[(size_t)i * nc + i];
      m.ry[i] = vy / M[(size_t)i * nc + i];
    }
    for (int i = nc - 1; i >= 0; i--) {
      double vx = m.rx[i], vy = m.ry[i];
      for (int q = i + 1; q < nc; q++) {
        vx -= M[(size_t)q * nc + i] * sx[q];
        vy -= M[(size_t)q * nc + i] * sy[q];
      }
      sx[i] = vx / M[(size_t)i * nc + i];
      sy[i] = vy / M[(size_t)i * nc + i];
    }
  }
  __syncthreads();
  return s_bad == 0;
}

// residual |sum of steps i..j-1 - measured| of row r (steps summed k ascending)
__device__ double row_residual(const SolveSmem& m, const double* wx, const double* wy, int r) {
  const int2 q = m.pr[r];
  double ax = 0.0, ay = 0.0;
  for (int k = q.x; k < q.y; k++) {
    ax += wx[k];
    ay += wy[k];
  }
  const double dx = ax - (double)m.ps[r].x, dy = ay - (double)m.ps[r].y;
  return sqrt(dx * dx + dy * dy);
}

size_t solve_smem_bytes(int P, int nf) {
  const size_t nc = nf - 1;
  return (size_t)P * (sizeof(int2) + sizeof(float2) + 2 * sizeof(int) + sizeof(double)) + nc * nf * sizeof(int) +
         (size_t)nf * sizeof(int) + nc * nc * sizeof(double) + 6 * (size_t)nf * sizeof(double) + 64;
}

}  // namespace

__global__ void __launch_bounds__(kSolveThreads) k_solve_smem(SolveArgs a) {
  extern __shared__ double sdyn[];
  const int P = a.npairs, nf = a.nframe, nc = nf - 1, tid = threadIdx.x;
  SolveSmem m;
  m.M = sdyn;
  m.rx = m.M + (size_t)nc * nc;
  m.ry = m.rx + nc;
  double* wx = m.ry + nc;
  double* wy = wx + nc;
  m.ki = wy + nc;
  m.ps = reinterpret_cast<float2*>(m.ki + P);
  m.pr = reinterpret_cast<int2*>(m.ps + P);
  m.mask = reinterpret_cast<int*>(m.pr + P);
  m.hist = m.mask + P;
  m.order = m.hist + (size_t)nc * nf;
  m.uf = m.order + P;
  for (int r = tid; r < P; r += kSolveThreads) {
    m.pr[r] = a.pairs[r];
    m.ps[r] = make_float2(a.pshift[2 * r], a.pshift[2 * r + 1]);
    m.mask[r] = 1;
  }
  __syncthreads();
  if (!solve_masked_smem(m, P, nf, wx, wy)) {
    if (tid == 0) *a.status = -6;
    return;
  }
  for (int r = tid; r < P; r += kSolveThreads) {
    const double v = row_residual(m, wx, wy, r);
    m.ki[r] = v;
    a.ki1[r] = v;
    m.order[r] = r;  // every slot holds a row even if NaN residuals share a rank
  }
  __syncthreads();
  // stable ascending rank of ki1 (OD_Threshold's repeated first-minimum pick)
  int* order = m.order;
  for (int r = tid; r < P; r += kSolveThreads) {
    const double v = m.ki[r];
    int pos = 0;
    for (int q = 0; q < P; q++) {
      const double u = m.ki[q];
      pos += (u < v || (u == v && q < r)) ? 1 : 0;
    }
    order[pos] = r;
  }
  __syncthreads();
  if (tid == 0) {
    int i;
    for (i = P - 1; i >= nc; i--)
      if (m.ki[order[i]] < (double)a.kithresh) break;
    int len = i + 1;
    int* par = m.uf;
    for (int f = 0; f < nf; f++) par[f] = f;
    int comps = nf;
    for (int q = 0; q < P; q++) m.mask[q] = 0;
    auto add = [&](int row) {
      m.mask[row] = 1;
      const int x = uf_find(par, m.pr[row].x), y = uf_find(par, m.pr[row].y);
      if (x != y) {
        par[x] = y;
        comps--;
      }
    };
    for (int q = 0; q < len && q < P; q++) add(order[q]);
    while (comps > 1 && len < P) add(order[len++]);
    *a.nkept = min(len, P);
  }
  __syncthreads();
  if (!solve_masked_smem(m, P, nf, wx, wy)) {
    if (tid == 0) *a.status = -6;
    return;
  }
  // kept rows ascending with their second-round residuals: an exclusive scan
  // of the mask gives each kept row its slot
  __shared__ int s_base;
  __shared__ int s_warp[kSolveThreads / 32];
  if (tid == 0) s_base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < P; c0 += kSolveThreads) {
    const int r = c0 + tid;
    const int f = (r < P && m.mask[r]) ? 1 : 0;
    const int lane = tid & 31, wid = tid >> 5;
    int incl = f;
    for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    int before = s_base;
    for (int w = 0; w < wid; w++) before += s_warp[w];
    if (f) {
      const int slot = before + incl - 1;
      a.kept[slot] = r;
      a.ki2[slot] = row_residual(m, wx, wy, r);
    }
    __syncthreads();
    if (tid == 0) {
      int t = 0;
      for (int w = 0; w < kSolveThreads / 32; w++) t += s_warp[w];
      s_base += t;
    }
    __syncthreads();
  }
  if (tid == 0) {
    double* sx = a.shift;
    double ox = 0.0, oy = 0.0, px = 0.0, py = 0.0, tx = 0.0, ty = 0.0;
    a.frame_shift[0] = 0.0;
    a.frame_shift[1] = 0.0;
    for (int k = 0; k < nc; k++) {
      const double nx = ox + wx[k], ny = oy + wy[k];
      ox = nx;
      oy = ny;
      const double stx = nx - px, sty = ny - py;
      px = nx;
      py = ny;
      sx[2 * k] = stx;
      sx[2 * k + 1] = sty;
      m.rx[k] = stx;  // shared copies for the sums below (no global reads back)
      m.ry[k] = sty;
      tx += stx;
      ty += sty;
      a.frame_shift[2 * (k + 1)] = tx;
      a.frame_shift[2 * (k + 1) + 1] = ty;
    }
    double mx = 0.0, my = 0.0;
    if (a.align_to_mid)
      for (int k = 0; k < a.mid_steps; k++) {
        mx += m.rx[k];
        my += m.ry[k];
      }
    double Tx = 0.0, Ty = 0.0;
    for (int k = 1; k < a.sum_first + 1; k++) {
      Tx += m.rx[k - 1];
      Ty += m.ry[k - 1];
    }
    for (int k = a.sum_first; k <= a.sum_last; k++) {
      if (k > a.sum_first) {
        Tx += m.rx[k - 1];
        Ty += m.ry[k - 1];
      }
      const int q2 = k - a.sum_first;
      a.sum_shift[q2] = make_double2(-Tx + mx, -Ty + my);
      a.sum_frames[q2] = k;
      a.sum_apply[q2] = (k == a.sum_first && !a.align_to_mid) ? 0 : 1;
    }
    // the final solve's per-step shifts into work[], where the host reads them
    for (int k = 0; k < nc; k++) {
      a.work[k] = wx[k];
      a.work[nc + k] = wy[k];
    }
    *a.status = 0;
  }
}

cudaError_t launch_solve(const SolveArgs& a, cudaStream_t st) {
  const size_t smem = solve_smem_bytes(a.npairs, a.nframe);
  if (smem <= 200 * 1024) {
    cudaError_t e = allow_smem((const void*)k_solve_smem, smem);
    if (e != cudaSuccess) return e;
    k_solve_smem<<<1, kSolveThreads, smem, st>>>(a);
    return cudaGetLastError();
  }
  k_solve<<<1, kSolveThreads, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace mc
