// Hand-written sm_100a kernels of the drift-correction path, in translation
// units that compile in parallel:
//   mc_fwd.cu, mc_fwd_raw.cu, mc_fwd_dif.cu   k_fwd_rows*, k_rows_fft*: decode +
//        dark/gain + crop + row R2C with transposed store (DFAlign.cu:710-806),
//        column FFT with Fourier-crop binning (cufunc.cu:162-176, 223-227)
//   mc_pair.cu   k_pair_cols*, k_pair_rows: cross power x B-factor + pruned
//        inverse FFTs onto the pbx window (cufunc.cu:229-233, 343-407)
//   mc_sum.cu    k_peak, k_shift_sum*, k_c2r_rows*, k_count_sum, k_objective
//        (cufunc.cu:372-497, DFAlign.cu:1287-1292)
//   this file    host helpers shared by all of them
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "kernels.cuh"

namespace mc {

// Raise-only, thread-safe opt-in to large dynamic shared memory.  The
// attribute is per function and per device; two host threads that launch
// the same kernel with different sizes must never lower it under each other.
cudaError_t allow_smem(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = done[{dev, func}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

}  // namespace mc
