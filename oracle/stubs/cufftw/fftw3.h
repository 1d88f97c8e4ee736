/* Test infrastructure: FFTW's single-precision API for the reference's full
 * program, answered by cuFFT's FFTW-compatible interface (libcufftw).  The
 * reference's host transforms (FindShift's 16x16 R2C and 512x512 C2R,
 * func.cpp:10-24) therefore run on the GPU through cuFFT with host buffers
 * in and out, instead of on the CPU through FFTW. */
#pragma once
#include <cufftw.h>
