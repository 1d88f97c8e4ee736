// Kernel argument blocks and launchers of libmc.
//
// Spectrum layout in HBM: one frame's half spectrum is stored column-major,
// spec[kx * ldn + ky] for kx in [0, n/2], ky in [0, n) (ky >= n/2 meaning
// ky - n), ldn = n rounded up to a multiple of 4 complex (32 bytes).  Every
// ky-column is contiguous, so the per-column work of the pair and sum stages
// reads whole 29.7 KB columns (n = 3710) with unit stride.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fft_engine.cuh"
#include "mc.h"

namespace mc {

// ---------------------------------------------------------------- forward --
// Pass A: decode + dark/gain + crop + row R2C of length nu, keeping kx < hk,
// written transposed: T[kx * ldt + y].
struct FwdRowsArgs {
  const void* frame;   // ny rows of nx pixels (MRC pixel type `mode`)
  // when set, the frame is *frames_slot + frame_offset bytes instead: the base
  // of the run's frames is read on the device, so a captured graph serves any
  // frame buffer written to the slot before its launch
  const void* const* frames_slot;
  long long frame_offset;
  int mode;            // 0 int8, 1 int16, 2 float32, 6 uint16
  int nx, ny;
  int offx, offy, nu;  // square crop
  int hk;              // kept kx columns (n/2 + 1)
  const float* dark;   // nx*ny or null
  const float* dark2;  // nx*ny or null (0 when dark given)
  const float* norm;   // nx*ny or null
  const float* norm2;  // nx*ny or null (1 when norm given)
  int two_outputs;     // 1: refs make hbuf != hbuf2, row y -> (outA, outB)
  float2* outA;
  float2* outB;
  int ldt;
  FftPlan1D plan;      // length nu, forward
  const float2* tw;    // nu twiddles exp(-2 pi i m / nu)
  int paired;          // radix-53 step: 0 built-in, 1 one output pair per loop pass, 2 two
};

// Pass B and every other batched transform over contiguous rows:
// out_row[i] = X[i] for i < keep_lo, X[i + n_in - n_out] otherwise.
struct RowsFftArgs {
  const float2* in;
  long long ld_in;
  float2* out;
  long long ld_out;
  int nrows;
  int n_out;
  int keep_lo;
  float scale;
  FftPlan1D plan;
  const float2* tw;
  int paired;          // radix-53 step: 0 built-in, 1 one output pair per loop pass, 2 two
};

// ------------------------------------------------------------------ pairs --
// Column stage: for pair p and column kx,
//   G[p][kx][m] = sum_ky c(ky) exp(+2 pi i ky y_m / n),  y_m = (ystart+m) mod n
//   c(ky) = A[kx][ky] conj(B[kx][ky]) exp(mbf*(kx^2+ky^2)) / ((n/2+1) n)
// evaluated with n = P*Q: Q-point inverse FFTs of the P stride-P subsequences
// followed by a P-term sum per output.
struct PairColsArgs {
  const float2* specA;
  long long strideA;   // elements between frames (0: one shared spectrum)
  const float2* specB;
  long long strideB;
  const int2* pairs;   // (frame of A, frame of B)
  int npairs;
  int pairs_per_cta;
  int n, ldn, H;
  float mbf;           // -0.5*bfactor/n/n as float
  float inv_size;      // 1 / ((n/2+1) n)
  int P, Q;
  FftPlan1D qplan;     // length Q
  const float2* twQ;   // Q twiddles exp(-2 pi i m / Q)
  const float2* twO;   // [P][box] exp(+2 pi i k1 y_m / n)
  const float2* twN;   // exp(+2 pi i e / n), n entries: when set (P*box > n), the generic
                       // kernel reads twO[k1][m] as twN[(k1 * y_m) mod n] (the same floats)
  int box;
  int ystart;
  float2* G;           // [npairs][H][box]
};

// Row stage: box[p][yb][xb] = sum_kx Re(G[p][kx][yb] * h(kx) exp(+2 pi i kx x_xb / n))
// with h = 1 at kx = 0, n/2 and 2 otherwise; cs[kx][xb] = h*(cos, sin).
struct PairRowsArgs {
  const float2* G;
  int npairs, H, box;
  const float2* cs;    // [H][box]
  float* boxes;        // [npairs][box][box]
  // when set with a compiled split n = P*Q: the pruned-transform row kernel
  // (twO and ystart as in PairColsArgs); otherwise the product kernel
  const float2* twO;
  int P, Q, ystart;
};

// Peak: integer argmax over the box, 16x16 sub-box, x32 Fourier upsampling,
// argmax on the 512x512 grid (all in FP64).
struct PeakArgs {
  const float* boxes;
  int npairs, box, n, nps;
  const double* w16;   // [16][9] cosine-mask weights
  float* shift;        // [npairs][2]
  float* cc;           // [npairs]
  int* peak;           // [npairs][2] integer box peak (x, y)
};

// -------------------------------------------------------------------- sum --
// sum_f spec_f[kx][ky] * exp(+2 pi i (sx_f kx + sy_f ky) / n) over a frame list.
// mode 0: write the sum spectrum out[kx*ld_out + ky].
// mode 1: inverse FFT along ky and write transposed t2[y*ld_t2 + kx].
struct ShiftSumArgs {
  const float2* spec;
  long long stride;
  const int* frames;     // positions of the summed frames
  const double2* shifts; // (sx, sy) per listed frame
  const int* apply;      // 1 = multiply by the phase ramp, 0 = add unshifted
  int nsum;
  int n, ldn, H;
  int mode;
  float2* out;
  long long ld_out;
  FftPlan1D plan;        // length n (mode 1)
  const float2* tw;
  float2* acc;           // mode 1: H x ldn scratch for the sum spectrum (split
                         // accumulate / transform); null = fused kernel
  int accumulate;        // mode 0: 1 = add the listed frames onto out's contents
                         // (a sum over several launches), 0 = overwrite
};

// FSC shell sums of -fsc over the listed frames (even / odd list positions).
struct FscArgs {
  const float2* spec;
  long long stride;
  const int* frames;
  const double2* shifts;  // sum shifts of the listed frames
  const int* apply;
  int nsum;
  int n, ldn, H;
  int step, nbox;          // shell width n/400 and shell count (n/2+1)/step + 1
  double dirx, diry;       // unit drift direction
  float edge;              // cos(pi/4) in float
  double* part;            // H x [2][nbox][6] per-column tables
  double* out;             // [2][nbox][6]: along / across drift; raw (x, aa, bb), corrected (x, aa, bb)
};

// C2R of rows y, y+1 packed as one complex inverse FFT: image[y][x] * scale.
struct C2rRowsArgs {
  const float2* t2;
  long long ld_t2;
  int n, H;
  float scale;
  float* image;          // n x n
  FftPlan1D plan;        // length n
  const float2* tw;
};

// Phase-ramp tables for the sum: ey[f][ky] = exp(+2 pi i sy_f ky_signed / n).
struct RampArgs {
  const double2* shifts;
  int nsum, n;
  float2* ey;            // [nsum][n]
};

// ---------------------------------------------------------------- adjoint --
// Frame-to-sum objective of the gradient refinement, for sum shifts s_k:
//   J = sum h w |S|^2,  S = sum_k F_k exp(+i w.s_k)   (S given, mode-0 sum)
//   g_k = -2 sum h w w_vec Im(u_k),  H_k = -2 sum h w w_vec w_vec^T Re(u_k),
//   u_k = conj(S - P_k) P_k,  P_k = F_k exp(+i w.s_k)
// h = half-spectrum multiplicity, w = exp(mbf r^2).  One CTA per column kx
// reads S and every frame's column once; FP64 partials per (kx, frame).
struct ObjectiveArgs {
  const float2* spec;
  long long stride;
  const int* frames;     // spectrum index of each listed frame (null: 0, 1, ...)
  int nframes;
  const float2* S;       // [kx][ky], pitch ldn
  const double2* shifts; // per frame (sx, sy)
  const float2* ey;      // [frame][ky] exp(+2 pi i sy ky / n) (k_ramp table)
  int n, ldn, H;
  float mbf;
  double* partial;       // [H][nframes][5]: gx, gy, hxx, hxy, hyy (without the -2)
  double* partialJ;      // [H]
  double* out;           // [nframes][5] (with the -2) then J at out[5*nframes]
};
cudaError_t launch_objective(const ObjectiveArgs& a, cudaStream_t st);

// ------------------------------------------------------------ device solve --
// Single-CTA FP64 drift solve + sum-shift preparation (mc_solve.cu).
struct SolveArgs {
  const int2* pairs;     // (i, j), i < j
  int npairs;
  const float* pshift;   // [P][2] measured pair shifts
  int nframe;
  float kithresh;
  int align_to_mid, mid_steps, sum_first, sum_last;
  // scratch
  double* M;             // [(nframe-1)^2]
  double* rhs;           // [2 (nframe-1)]
  double* work;          // [2 (nframe-1) + 2 nframe]
  int* mask;             // [P]
  int* order;            // [P]
  int* uf;               // [nframe]
  // outputs
  double* ki1;           // [P]
  int* kept;             // [P] kept rows, ascending (first *nkept valid)
  int* nkept;
  double* ki2;           // [P] residuals of the kept rows
  double* shift;         // [nframe-1][2] per-step shifts
  double* frame_shift;   // [nframe][2]
  double2* sum_shift;    // [sum_last - sum_first + 1]
  int* sum_frames;
  int* sum_apply;
  int* status;           // 0 ok, -6 singular system
};
cudaError_t launch_solve(const SolveArgs& a, cudaStream_t st);
cudaError_t launch_ramp(const double2* shifts, int nsum, int n, float2* ey, cudaStream_t st);

// Exact integer sum of raw frames over the square crop (A1 count sums):
// out[y*nu + x] = sum_f frame_f[offy + y][offx + x] for f in [first, last],
// pixels decoded as the reference does (mode 0 signed char, 1 int16, 6 uint16).
struct CountSumArgs {
  const void* frames;    // run positions back to back, nx*ny pixels each
  long long frame_pixels;
  int mode, nx, offx, offy, nu;
  int first, last;       // run positions
  int* out;              // nu*nu
};
cudaError_t launch_count_sum(const CountSumArgs& a, cudaStream_t st);

cudaError_t launch_fwd_rows(const FwdRowsArgs& a, cudaStream_t st);
cudaError_t launch_rows_fft(const RowsFftArgs& a, bool inverse, int rows_per_cta, cudaStream_t st);
cudaError_t launch_pair_cols(const PairColsArgs& a, cudaStream_t st);
cudaError_t launch_pair_rows(const PairRowsArgs& a, cudaStream_t st);
cudaError_t launch_peak(const PeakArgs& a, cudaStream_t st);
// ey: scratch of nsum*n float2 for the per-frame ky phase ramps
cudaError_t launch_shift_sum(const ShiftSumArgs& a, float2* ey, cudaStream_t st);
int shift_sum_kernels(const ShiftSumArgs& a);  // kernels launch_shift_sum launches
// n = N1 * N2 for one of the compiled two-level splits
bool two_level_split(int n, int& n1, int& n2);
cudaError_t launch_c2r_rows(const C2rRowsArgs& a, cudaStream_t st);
// -scx/-scy stretch: the crop region of one raw frame (word length wl, read
// through `slot` + offset when slot is set, else from `frame`) gathered into
// the same region of the full-size frame dst; and a whole float reference.
cudaError_t launch_stretch_crop(const void* const* slot, long long offset, const void* frame, int wl, void* dst,
                                const int* rmap, const int* cmap, int nx, int offx, int offy, int nu,
                                cudaStream_t st);
cudaError_t launch_stretch_full(const float* src, float* dst, const int* rmap, const int* cmap, int nx, int ny,
                                cudaStream_t st);
// ey: scratch of nsum*n float2 (the ky phase ramps of the listed frames)
cudaError_t launch_fsc(const FscArgs& a, float2* ey, cudaStream_t st);
size_t fsc_smem(int nbox, int nsum);

// ------------------------------------------------------------ quick-look --
// Displays of -dsp 1 (DFAlign.cu:73-178, 841-849, 1270-1286; func.cpp:459-556).
// Log modulus of a half spectrum spec[kx*ldn + ky] laid out as the centred
// n x n display image of FFTModulusToDispBuf: column c >= n/2 holds kx = c - n/2,
// row r holds ky = r + n/2 (r < n/2) or r - n/2; the left half mirrors the
// right through the centre, row 0's left half repeats row 1's.
cudaError_t launch_ql_logmod(const float2* spec, int ldn, int n, float scale, float* img, cudaStream_t st);
// Fourier crop of a half spectrum [kx][ky] (ld ldn, side n) to side d:
// out[kx*d + k] for kx <= d/2, k < d/2 from ky = k, else from ky = n - d + k.
cudaError_t launch_ql_crop(const float2* spec, int ldn, int n, int d, float2* out, cudaStream_t st);
// Unnormalised C2R of a side-d half spectrum in[kx*d + ky] (kx <= d/2):
// img[y*d + x] = scale * sum_kx h(kx) Re(exp(+2 pi i kx x/d) sum_ky in exp(+2 pi i ky y/d)),
// h = 1 at kx = 0, d/2, else 2; tmp holds (d/2+1) x d complex.
cudaError_t launch_ql_c2r(const float2* in, int d, float scale, float2* tmp, float* img, cudaStream_t st);

// Sets the calling thread's mc_last_error() text; returns `code`.
int record_error(int code, const char* text);

// Opt-in to `bytes` of dynamic shared memory for `func` on the current device;
// never lowers an earlier, larger opt-in (safe with concurrent host threads).
cudaError_t allow_smem(const void* func, size_t bytes);

// true when the register-codelet column stage handles the split n = P*Q
bool pair_cols_reg_supported(int P, int Q);
// the split n = P*Q a plan's register-codelet column stage uses for (n, box)
// (schedule or cost model); false when n has none (mc_plan.cu)
bool reg_pair_split(int n, int box, int* P, int* Q);
size_t pair_cols_reg_smem(int n, int team);
// dynamic shared memory launch_pair_cols asks for with this split
size_t pair_cols_launch_smem(int n, int P, int Q, int box);

size_t fwd_rows_smem(int nu);
size_t rows_fft_smem(int n, int rows_per_cta);
size_t pair_cols_smem(int n, int P, int Q, int box);
// the generic column kernel keeps a length-n twiddle table instead of P x box
inline bool pair_cols_tabn(int n, int P, int box) { return (long long)P * box > n; }
size_t shift_sum_smem(int n, int nsum);
size_t c2r_rows_smem(int n);
size_t peak_smem();

}  // namespace mc
