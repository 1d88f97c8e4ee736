/* Test-infrastructure stand-in for FFTW's public header (the single-precision
 * names the reference's func.cpp declares against).  Only lets func.cpp
 * compile so that its FFT-free functions can be called from
 * oracle/ref_func_harness.cpp; the plan functions abort if ever reached. */
#pragma once
typedef float fftwf_complex[2];
typedef struct fftwf_plan_s* fftwf_plan;
#define FFTW_ESTIMATE (1U << 6)
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
