/*
 * libmc -- B200-native drift correction of dose-fractionated movies.
 *
 * C ABI of the frame-drift correction path of MotionCorr 1
 * (dosefgpu_driftcorr, gepeng1983/motioncorr1exp, src-1125).  It replaces
 * the reference's GPU layer (cufunc.h:16-47) and the body of
 * CDFAlign::ThreadFunc_cuAlign (DFAlign.cu:456-1355): the caller reads the
 * stack and writes the outputs, the library does everything in between on
 * one GPU with hand-written sm_100a kernels (no cuFFT).
 *
 * Conventions
 *   - every call returns MC_OK (0) or a negative MC_E_* code; mc_strerror()
 *     and mc_last_error() describe it; nothing exits or installs handlers;
 *   - the caller owns host buffers, a plan owns its device memory and its
 *     CUDA stream; a plan is used by one host thread at a time and distinct
 *     plans share no state;
 *   - "position" p means frame nStart + p of the stack (0 <= p < nframe).
 */
#ifndef MC_H
#define MC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MC_VERSION 10000 /* 1.0.0 */

/* Pixel modes a plan decodes on the GPU: the MRC modes 0 (signed 8-bit, as
 * read2DIm_32bit converts char, mrc.cpp:338-348), 1 (int16), 2 (float32),
 * 6 (uint16), and MC_MODE_U8: unsigned 8-bit pixels, as 8-bit TIFF strips
 * hold them (MRCT::read2DIm converts unsigned char, mrct.cpp:137-150).
 * 16-bit TIFF strips are mode 6.  Added (no reference counterpart):
 * MC_MODE_F16, the MRC2014 mode 12 of IEEE-754 half floats -- frames stored
 * in half the bytes of mode 2 and widened to FP32 in the forward kernels'
 * loads; integer counts up to 2048 convert to it exactly. */
#define MC_MODE_U8 100
#define MC_MODE_F16 12

enum {
  MC_OK = 0,
  MC_E_ARG = -1,      /* invalid argument / parameter combination */
  MC_E_CUDA = -2,     /* CUDA runtime error (see mc_last_error) */
  MC_E_NOMEM = -3,    /* device or host allocation failed */
  MC_E_SIZE = -4,     /* geometry the kernels do not support */
  MC_E_STATE = -5,    /* call out of order (e.g. pairs before forward) */
  MC_E_NUMERIC = -6,  /* singular least-squares system */
  MC_E_IO = -7        /* stack file missing, unreadable, malformed or of an unsupported kind */
};

/* Alignment parameters: the fields of APARA (DFAlign.h:16-63) that act on the
 * drift-correction path, plus -itr/-ith (DFAlign.h:75-76) and the added
 * refinement switch.  Defaults: mc_default_params. */
typedef struct mc_params {
  int crop_offsetx;    /* -crx */
  int crop_offsety;    /* -cry */
  int crop_nsam;       /* -crd (0 = largest square) */
  float bin;           /* -bin, clamped to [1, 2] */
  int nStart;          /* -nst */
  int nEnd;            /* -ned */
  int nStartSum;       /* -nss */
  int nEndSum;         /* -nes */
  int GPUNum;          /* -gpu */
  float bfactor;       /* -bft, pix^2 */
  int CCPeakSearchDim; /* -pbx, 16..256 */
  int FrameDistOffset; /* -fod */
  int NoisePeakSize;   /* -nps */
  float kiThresh;      /* -kit */
  int bAlignToMid;     /* -atm */
  int iter;            /* -itr */
  float iterthres;     /* -ith */
  int refine;          /* added: 0 = Fourier-upsampled peak only, 1 = + gradient refinement */
} mc_params;

typedef struct mc_plan mc_plan;

typedef struct mc_info {
  int nx, ny, nz, mode;  /* stack geometry and pixel mode (0, 1, 2, 6, MC_MODE_U8) */
  int nsam_unbin;        /* square crop side (verifyCropSize, func.cpp:80-103) */
  int nsam;              /* binned side (DFAlign.cu:515) */
  int nstart, nend, nframe;
  int npairs;            /* frame pairs of OD_SetEquation_All (mfunc.h:64-84) */
  int two_sets;          /* 1 when dark/gain references make hbuf != hbuf2 */
  int prune_p, prune_q;  /* n = P*Q split of the pruned inverse transform */
  size_t device_bytes;   /* device memory held by the plan */
  int spectrum_slots;    /* 0: every frame's spectrum stays in HBM; else the
                            number of spectra held (mc_plan_create_slots) */
  long long forward_recomputes; /* forward transforms run again because their
                            spectrum had been given up (slot mode), since creation */
} mc_info;

typedef struct mc_timings { /* device time of the last run, CUDA events */
  float forward_ms, pairs_ms, solve_ms, iterate_ms, sum_ms, total_ms, refine_ms;
} mc_timings;

typedef void (*mc_log_fn)(const char* text, void* user);

int mc_version(void);
const char* mc_strerror(int code);
/* Text of the last error of the calling thread ("" if none). */
const char* mc_last_error(void);
/* Fault injection for tests (no reference counterpart): the nth device or
 * pinned-host allocation a plan makes from now on, in any thread, fails with
 * MC_E_NOMEM as if memory were exhausted; the countdown then disarms.
 * 0 disarms it.  The failure is simulated on the host, nothing is asked of
 * the GPU. */
void mc_debug_fail_alloc(int nth);
/* Test hook (no reference counterpart): plans created from now on see at
 * most `bytes` of free device memory when they size their spectrum store
 * (mc_plan_create_slots with slots = 0).  0 restores the real figure. */
void mc_debug_device_budget(size_t bytes);

/* getDefaultPara (dosefgpu_driftcorr.cpp:8-58) plus itr=0, ith=0 (DFAlign.cu:15-16). */
void mc_default_params(mc_params* p);

/* VerifyPara frame-range repair and checks (dosefgpu_driftcorr.cpp:60-118)
 * for a stack of nz frames.  Returns MC_E_ARG with the reference's abort text
 * in mc_last_error() when the reference aborts. */
int mc_verify_params(mc_params* p, int nz);

/* Plan for one stack geometry: crop/bin (DFAlign.cu:500-530), frame range,
 * device buffers, FFT plans.  Replaces initGPU, GPUMemAlloc, GPUFFTPlan,
 * GPUIFFTPlan and MkPosList (cufunc.cu:30-65, 111-115, 202-215, 309-341). */
int mc_plan_create(const mc_params* p, int nx, int ny, int nz, int mode, mc_plan** out);
void mc_plan_destroy(mc_plan* plan);
int mc_plan_info(const mc_plan* plan, mc_info* info);
/* The plan's CUDA stream (cudaStream_t). */
void* mc_plan_stream(mc_plan* plan);
/* Log sink for the text ThreadFunc_cuAlign writes through TextOutput
 * (DFAlign.cu:59-71); NULL disables. */
void mc_plan_set_log(mc_plan* plan, mc_log_fn fn, void* user);

/* Dark/gain references, nx*ny floats each, host memory, NULL = absent
 * (DFAlign.cu:614-695): dark2/norm2 are the second frames of two-frame
 * reference files; with a one-frame file pass NULL (then 0 / 1 are used). */
int mc_plan_set_refs(mc_plan* plan, const float* dark, const float* dark2, const float* norm,
                     const float* norm2);

/* Anisotropic magnification correction of -scx/-scy (DFAlign.cu:503-504,
 * 751-765), for the forward transforms of later runs: with r = 1/yscale and
 * c = 1/xscale in float, each dark/gain-corrected pixel (y, x) with y, x >= 1
 * takes the value at (int(y*r + 0.5), int(x*c + 0.5)) (float product, double
 * sum, nearest neighbour); row 0 and column 0 keep theirs.  Factors >= 1
 * (MC_E_ARG otherwise, with the reference's message); 1, 1 switches it off.
 * The exact count sums stay on the unstretched pixels. */
int mc_plan_set_stretch(mc_plan* plan, float xscale, float yscale);

/* Copy raw frames (MRC pixel type of the plan's mode, nx*ny each) for
 * positions [first, first+count) from host memory (pinned or pageable) or
 * from device memory.  Replaces MRC::read2DIm_32bit + GPUMemH2D per frame
 * (DFAlign.cu:713, 770, 795).  Host copies return once the source buffer
 * may be reused; device copies are ordered on the plan stream, which does
 * not wait for the caller's streams: the frames must be complete when the
 * call is made (synchronise the stream that wrote them). */
int mc_plan_load_frames(mc_plan* plan, const void* frames, int first, int count);
int mc_plan_load_frames_device(mc_plan* plan, const void* d_frames, int first, int count);

/* Stages (each synchronous on return). */
int mc_plan_forward(mc_plan* plan);         /* DFAlign.cu:710-824 */
int mc_plan_pairs(mc_plan* plan);           /* DFAlign.cu:875-905 */
int mc_plan_solve(mc_plan* plan);           /* DFAlign.cu:914-948 */
int mc_plan_iterate(mc_plan* plan);         /* DFAlign.cu:950-1092 */
int mc_plan_sum(mc_plan* plan, float* image_host); /* DFAlign.cu:1114-1292; image n*n or NULL */
/* All stages in order. */
int mc_plan_run(mc_plan* plan, float* image_host);
/* All stages in order on frames in host memory (all positions, file pixel
 * type): the upload runs in chunks on a second stream and overlaps the
 * forward transforms of the chunks already resident (pinned memory for the
 * overlap; pageable works but serialises).  Replaces the per-frame
 * read/GPUMemH2D/GPUFFT2d sequence of DFAlign.cu:710-820 plus the rest of
 * the path. */
int mc_plan_run_host(mc_plan* plan, const void* frames, float* image_host);

/* Results. */
int mc_plan_get_frame_shifts(const mc_plan* plan, double* xy);           /* 2*nframe, "Shift of Frame" */
int mc_plan_get_pairs(const mc_plan* plan, int* ij, float* shift, float* cc, int* peak); /* 2P,2P,P,2P */
int mc_plan_get_ki(const mc_plan* plan, double* ki1, int* nkept, int* kept, double* ki2);
int mc_plan_get_frame_means(const mc_plan* plan, float* mean);           /* nframe */
int mc_plan_get_spectrum(mc_plan* plan, int set, int pos, void* host);  /* (n/2+1)*n float2, [kx][ky] */
int mc_plan_get_boxes(mc_plan* plan, float* host);                       /* npairs*pbx*pbx */
int mc_plan_get_sum_shifts(const mc_plan* plan, double* xy, int* first, int* last);
int mc_plan_get_timings(const mc_plan* plan, mc_timings* t);

/* Added method (no reference counterpart; replaces the 1/32-px grid peak of
 * FindShift, cufunc.cu:457-481, as the final sub-pixel step).  Objective of
 * the frame-to-sum correlation for sum shifts s_k (the shifts
 * phase-shift-and-sum applies, s_k = -frameshift_k + const):
 *   J = sum_w h w |S|^2,  S = sum_k F_k exp(+i w.s_k),  w = B-factor weight,
 * its gradient dJ/ds_k (2*nframe) from the hand-written adjoint of the
 * shift-and-sum (one pass reading every spectrum once) and the 2x2 Hessian
 * blocks (3*nframe: xx, xy, yy).  Any output may be NULL. */
int mc_plan_objective(mc_plan* plan, const double* shifts_xy, double* J, double* grad, double* hess);
/* Block-Newton ascent of J from the peak-fit shifts (after mc_plan_iterate);
 * updates the final shifts.  mc_plan_run calls it when params.refine = 1. */
int mc_plan_refine(mc_plan* plan, int iterations);

/* Per-kernel accounting of a plan: launches and algorithmic bytes are always
 * counted; device time is recorded with one CUDA event pair per launch while
 * profiling is on.  Kinds follow the kernels of the path. */
enum {
  MC_K_FWD_ROWS = 0,  /* decode + dark/gain + crop + row R2C */
  MC_K_FWD_COLS = 1,  /* column FFT + Fourier-crop binning (k_rows_fft) */
  MC_K_PAIR_COLS = 2, /* cross power x B-factor + pruned inverse along ky */
  MC_K_PAIR_ROWS = 3, /* pruned C2R along kx onto the pbx window */
  MC_K_PEAK = 4,      /* integer + x32 Fourier-upsampled peak */
  MC_K_SHIFT_SUM = 5, /* phase-shift-and-accumulate (+ inverse columns) */
  MC_K_C2R_ROWS = 6,  /* final C2R rows x 1/n^2 */
  MC_K_OBJECTIVE = 7, /* adjoint of the shift-and-sum: objective, gradient, Hessian blocks */
  MC_K_SOLVE = 8,     /* FP64 drift solve of a device-only movie (k_solve_smem / k_solve) */
  MC_KERNEL_KINDS = 9
};
void mc_plan_set_profiling(mc_plan* plan, int on);
int mc_plan_reset_stats(mc_plan* plan);
int mc_plan_kernel_stats(const mc_plan* plan, int kind, double* ms, long long* launches, double* bytes);
const char* mc_kernel_name(int kind);

/* Host-only drift solve of DFAlign.cu:914-948 on given pair measurements:
 * lsSolver, residuals ki, OD_Threshold (mfunc.h:101-146), lsSolver again.
 * ij: 2*npairs frame indices (i < j), shifts_xy: 2*npairs; outputs step_xy
 * (2*(nframe-1) per-step shifts), ki1 (npairs), kept rows (ascending) and
 * their second-round residuals ki2.  Any output may be NULL. */
int mc_solve_pairs(int nframe, int npairs, const int* ij, const float* shifts_xy, float kithresh,
                   double* step_xy, double* ki1, int* nkept, int* kept, double* ki2);

/* No counterpart in the reference.  For callers that must not allocate
 * device memory -- code inside a detector's acquisition/streaming loop that
 * owns a fixed, pre-reserved memory budget, or a host framework that forbids
 * allocation once its own pool is set up: the pbx x pbx cross-correlation
 * window of one frame pair, the same window a plan's pair stage stores for
 * that pair (mc_plan_get_boxes), computed with no cudaMalloc/cudaFree and
 * no allocating library call.  Inputs: two half spectra already on the
 * device in this library's layout (spec[kx*ldn + ky], kx <= n/2, ky < n);
 * output: d_window, pbx*pbx floats on the device.  Intermediate data lives in
 * a 5 MiB file-scope device array that every GPU loading libmc holds until
 * exit.  Limits: n even in [16, 4096], pbx in [16, min(128, n)], n = P*Q with
 * P <= 128 and Q a register-codelet length; larger problems return MC_E_SIZE.
 * The first call on a device looks up the array's address on that device
 * (make it before any stream capture).  All calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller. */
int mc_pair_window_static(const void* d_spec_a, const void* d_spec_b, int n, int ldn, int pbx, float bfactor,
                          float* d_window, void* stream);

/* Extra outputs of the sum stage.  Images are nsam*nsam floats (host).
 * mc_plan_raw_sum: the unaligned sum of frames nStartSum..nEndSum, the
 *   "-srs" output (raw sums DFAlign.cu:807-813, transform and scale
 *   :851-858); needs mc_plan_forward (or a whole run).
 * mc_plan_sum_to: the aligned sum of frames nStartSum..last_frame with the
 *   final shifts, the "-2es" second sum (DFAlign.cu:1117-1122, 1198-1208;
 *   last_frame is an absolute frame number, clamped as the reference does);
 *   needs mc_plan_sum or mc_plan_run.
 * mc_plan_corrected_frame: one aligned frame of the "-ssc" corrected stack
 *   (DFAlign.cu:1154-1163, 1185-1195; absolute frame number in
 *   [nStartSum, nEndSum]); needs mc_plan_sum or mc_plan_run. */
int mc_plan_raw_sum(mc_plan* plan, float* image_host);
int mc_plan_sum_to(mc_plan* plan, int last_frame, float* image_host);
int mc_plan_corrected_frame(mc_plan* plan, int frame, float* image_host);

/* Quick-look displays of -dsp 1 (DFAlign.cu:73-178, 841-849, 1270-1286;
 * func.cpp:372-556): MC_QUICKLOOK_DIM^2 int16 pixels with values 0..255 (the
 * reference writes them as mode-1 MRC files in dosef_quick/).
 *   which 0: "RawFFT"  log(1 + 1e-4 |unaligned sum spectrum|) as the centred
 *            modulus image, Fourier-binned to 400 x 400;
 *   which 1: "CorrSum" the corrected sum, Fourier-binned to 400 x 400;
 *   which 2: "CorrFFT" as 0 for the corrected sum.
 * Contrast: 0.5 % histogram tails clipped, then linear to 0..255.  Needs a
 * binned side of at least 400; 0 needs mc_plan_forward, 1 and 2 a finished
 * sum (mc_plan_sum or mc_plan_run). */
#define MC_QUICKLOOK_DIM 400

/* FSC of -fsc (CDFAlign::PlotFSC, DFAlign.cu:212-326) from the resident
 * spectra and the current sum shifts: the summed frames split into even and
 * odd positions, unaligned (Raw) and aligned (Corr), correlated per Fourier
 * shell of width nsam/400 (nsam >= 400, else MC_E_SIZE), separately along
 * the drift of the last summed frame (D, |cos| > cos 45 deg) and across it
 * (U).  Fills min(cap, *nbox) rows of 5 doubles: Nq%, D_Raw, U_Raw, D_Corr,
 * U_Corr; *nbox = (nsam/2+1)/(nsam/400) + 1 (rows NULL: only this size,
 * nothing computed).  Shell sums in FP64 (the reference accumulates in
 * float). */
int mc_plan_fsc(mc_plan* plan, double* rows, int cap, int* nbox);
int mc_plan_quicklook(mc_plan* plan, int which, int16_t* out);

/* No counterpart in the reference (its raw sums are FP32 spectra): the
 * exact integer sum of the raw pixels of frames nStartSum..nEndSum over the
 * square crop, nsam_unbin*nsam_unbin int32 values (host), pixels decoded as
 * read2DIm_32bit does (mode 0 signed char, 1 int16, 6 uint16; mode 2 is
 * rejected).  Needs the frames loaded or bound. */
int mc_plan_count_sum(mc_plan* plan, int32_t* host_counts);

/* Batched 1-D complex FFT of the library's engine on device memory
 * (un-normalised; inverse = exp(+2 pi i)).  Stream may be NULL. */
int mc_fft1d(int n, int batch, int inverse, const void* d_in, void* d_out, void* stream);

/* ---------------------------------------------------------------- batching --
 * No counterpart in the reference, which aligns one movie per process
 * (dosefgpu_driftcorr.cpp:121-515).  These entry points serve many movies
 * from one process without reallocating per movie. */

/* Re-targets a plan at another frame range / stack depth of the same
 * geometry (crop, bin, pbx, bft, nps and GPU must match the plan's; nStart,
 * nEnd, nStartSum, nEndSum, fod, kit, atm, itr, ith and refine may change).
 * The new range must fit the plan's capacity (mc_plan_create_capacity).
 * Frames must be loaded or bound again afterwards. */
int mc_plan_reframe(mc_plan* plan, const mc_params* p, int nz);

/* mc_plan_create with device buffers sized for up to cap_frames aligned
 * frames and cap_pairs frame pairs (0 = this run's counts). */
int mc_plan_create_capacity(const mc_params* p, int nx, int ny, int nz, int mode, int cap_frames, int cap_pairs,
                            mc_plan** out);

/* mc_plan_create_capacity with a bound on the spectra held in HBM.  The
 * reference keeps every frame's spectrum in host memory and streams pairs
 * through the GPU (hbuf / hbuf2, DFAlign.cu:545-546); a plan keeps them in
 * HBM, and when a movie's spectra do not fit it holds `slots` of them and
 * recomputes a frame's forward transform from the raw frames (which stay in
 * HBM) whenever a stage needs a spectrum it gave up: the pair stage runs in
 * blocks of slots/2 frames against each other, the sums, iterations and the
 * refinement objective (its adjoint pass included) in chunks of `slots`
 * frames.  Results are those of the resident plan (the same kernels on the
 * same spectra, sums accumulated in the same frame order).
 *   slots = 0        : automatic -- every spectrum when the free device
 *                      memory allows it (keeping 256 MiB free), else as many
 *                      as fit; mc_plan_create and _capacity behave this way
 *   slots >= frames  : every spectrum resident
 *   4 <= slots       : at most `slots` spectra
 * Slot mode runs the host-driven pipeline (no captured movie graph) and has
 * no FSC (mc_plan_fsc returns MC_E_STATE). */
int mc_plan_create_slots(const mc_params* p, int nx, int ny, int nz, int mode, int cap_frames, int cap_pairs,
                         int slots, mc_plan** out);

/* Reads the run's frames (positions nStart..nEnd, nx*ny pixels each in the
 * plan's MRC mode, back to back) in place from caller device memory on the
 * plan's GPU instead of the plan's own frame buffer; the memory must stay
 * valid and unchanged until the run returns, and complete when the run
 * starts (the plan stream does not wait for the caller's streams).  NULL
 * unbinds.  A later
 * mc_plan_load_frames* or mc_plan_run_host switches back to the plan's
 * buffer. */
int mc_plan_bind_frames_device(mc_plan* plan, const void* d_frames);

/* Pair-stage schedule for one binned side n, as chosen by the autotuner
 * (motioncorr1exp_b200/autotune.py): process-wide, read by plans created
 * afterwards. */
typedef struct mc_schedule {
  int n;             /* binned side the entry applies to */
  int pair_q;        /* codelet length Q of the split n = P*Q (0 = built-in cost model) */
  int pairs_per_cta; /* pairs per CTA of the pair column stage (0 = 32) */
  int pair_variant;  /* reserved: 0 (the register-codelet column kernel) */
  int fwd_streams;   /* forked streams of the forward transforms, 1..8 (0 = 4) */
  int fwd_rows_pairing; /* radix-53 step of the forward row pass: 0 built-in, 1 one output pair */
  int fwd_cols_pairing; /* per loop pass, 2 two; likewise the column pass */
} mc_schedule;
int mc_schedule_set(const mc_schedule* s); /* replaces the entry for s->n */
int mc_schedule_get(int n, mc_schedule* out); /* MC_E_ARG when none is set */
void mc_schedule_clear(void);
/* Codelet lengths Q the pair column stage accepts for side n; returns the
 * count (at most max written to q_out). */
int mc_schedule_candidates(int n, int* q_out, int max);

typedef struct mc_batch mc_batch;

typedef struct mc_batch_job {
  const void* frames;    /* the run's frames (positions nStart..nEnd), back to back */
  int on_device;         /* 1: frames is device memory of params.GPUNum, read in place */
  int nx, ny, nz, mode;  /* stack geometry and MRC pixel mode */
  mc_params params;      /* as mc_verify_params left them; no dark/gain references */
  float* image;          /* out: nsam*nsam host floats, or NULL */
  double* frame_shifts;  /* out: 2*nframe host doubles ("Shift of Frame"), or NULL */
} mc_batch_job;

typedef struct mc_batch_result {
  int status;            /* MC_OK or the movie's error code */
  int nsam, nframe, npairs;
  int lane;              /* lane that ran the movie */
  double start_ms;       /* host clock, from the start of mc_batch_run */
  double end_ms;         /* results on the host */
  float gpu_ms;          /* device time of the movie (CUDA events) */
  char message[160];     /* mc_last_error() text of a failed movie */
} mc_batch_result;

/* A batch runner with `lanes` worker threads on one GPU, each with its own
 * stream and its own plans (one per stack geometry, kept across runs and
 * replayed as CUDA graphs per frame configuration). */
int mc_batch_create(int device, int lanes, mc_batch** out);
void mc_batch_destroy(mc_batch* b);
/* Aligns every job; lanes take jobs in order from a shared queue.  Returns
 * MC_OK when every movie succeeded, else the first failing movie's code
 * (the others still run; see results[i].status). */
int mc_batch_run(mc_batch* b, const mc_batch_job* jobs, int njobs, mc_batch_result* results);
/* Device memory held by the runner's plans. */
size_t mc_batch_device_bytes(const mc_batch* b);
/* Single-graph mode (on = 1): mc_batch_run captures the whole batch -- every
 * movie's forward transforms, pair stage, FP64 solve, sum and C2R, lane l
 * taking jobs l, l + lanes, ... as its own branch -- into one CUDA graph,
 * launches it once and reads every movie's results after one
 * synchronisation; the graph is kept and relaunched while the job list is
 * the same.  Every job must hold device frames (on_device = 1), run
 * device-only (-itr 0, no refinement) and give its image in pinned host or
 * device memory (or NULL); otherwise mc_batch_run returns MC_E_ARG.  A
 * movie whose plan holds spectrum slots (its spectra did not fit the free
 * device memory; mc_plan_create_slots) gives MC_E_STATE: run such batches
 * with lanes.  The per-movie gpu_ms is 0 and start/end times are the
 * batch's.  No reference counterpart (the reference aligns one movie per
 * process). */
int mc_batch_set_graph(mc_batch* b, int on);

/* ---- Stack files (host only; no GPU needed) -------------------------------
 * One handle over the three stack formats: replaces the readers MRC, MRCZ
 * and MRCT (mrc.cpp:29-157, 325-382; mrcz.cpp:23-110; mrct.cpp:29-152) and
 * the detection order of the alignment thread (DFAlign.cu:470-479): TIFF by
 * its byte-order mark (isTIFF, func.cpp:608-627), MRC-gz by the gzip magic
 * plus the 'MAP ' stamp of the inflated header (isMRCZ, func.cpp:580-606),
 * MRC by the stamp or a file name containing "mrc" (isMRC, func.cpp:557-578).
 * TIFF: one image per directory, 8- or 16-bit, one sample, strips (no
 * tiles), compression none, LZW, Deflate or PackBits, predictor 1 or 2,
 * classic or BigTIFF, either byte order; no libtiff is linked. */
typedef struct mc_stack mc_stack;
enum { MC_STACK_MRC = 0, MC_STACK_MRCZ = 1, MC_STACK_TIFF = 2 };
typedef struct mc_stack_info {
  int nx, ny, nz;
  int mode;         /* pixel mode of the raw frames below: the MRC mode, or
                       MC_MODE_U8 / 6 for 8- / 16-bit TIFF (mc_plan_create's mode) */
  int file_mode;    /* the mode the reference reports: the MRC header's, 7199 for
                       TIFF (fakeReadHeader, mrct.cpp:104-123) */
  int format;       /* MC_STACK_* */
  int bits;         /* bits per pixel */
  int compression;  /* TIFF Compression tag (1, 5, 8, 32773, 32946); 0 for MRC */
} mc_stack_info;
/* MC_E_IO (message in mc_last_error) when the file is none of the three or
 * holds a variant this reader does not decode. */
int mc_stack_open(const char* path, mc_stack** out);
int mc_stack_get_info(const mc_stack* s, mc_stack_info* info);
/* Raw pixels of frames [first, first+count) back to back into dst
 * (nx*ny*word length bytes each; TIFF directory k is frame k).  TIFF frames
 * decode in parallel on host threads.  *got (may be NULL) = the leading
 * frames read; MC_E_IO when fewer than count.  Replaces read2DIm
 * (mrc.cpp:151-157, mrcz.cpp:103-109, mrct.cpp:113-152). */
int mc_stack_read_frames(mc_stack* s, void* dst, int first, int count, int* got);
/* Frame n converted to float as read2DIm_32bit does (mrc.cpp:325-382; TIFF
 * bytes and words unsigned, mrct.cpp:137-150). */
int mc_stack_read_frame_float(mc_stack* s, float* dst, int n);
void mc_stack_close(mc_stack* s);

#ifdef __cplusplus
}
#endif
#endif /* MC_H */
