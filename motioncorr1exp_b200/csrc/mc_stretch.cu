// Anisotropic magnification correction of -scx/-scy (DFAlign.cu:751-765):
// nearest-neighbour stretch of each dark/gain-corrected frame, pixel (Y, X)
// with Y, X >= 1 taking the value at (rmap[Y], cmap[X]), row 0 and column 0
// unchanged.  The maps (int(Y * (1/yscale) + 0.5) in the reference's float
// then double arithmetic) come from the host.  Because the correction is
// pointwise, gathering the raw pixels and the references through the same
// map gives exactly the corrected value at the source pixel.
#include "kcommon.cuh"

namespace mc {
namespace {

__device__ __forceinline__ long long stretch_src(int Y, int X, int nx, const int* __restrict__ rmap,
                                                 const int* __restrict__ cmap) {
  if (Y == 0 || X == 0) return (long long)Y * nx + X;
  return (long long)rmap[Y] * nx + cmap[X];
}

// The crop region [offy, offy+nu) x [offx, offx+nu) of one raw frame, in
// place in a full-size frame buffer (the forward kernels read only there).
template <typename W>
__global__ void k_stretch_crop(const void* const* slot, long long offset, const void* frame, W* dst,
                               const int* __restrict__ rmap, const int* __restrict__ cmap, int nx, int offx,
                               int offy, int nu) {
  const W* src = reinterpret_cast<const W*>(slot ? static_cast<const char*>(*slot) + offset
                                                 : static_cast<const char*>(frame));
  const long long total = (long long)nu * nu;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(t / nu), x = (int)(t - (long long)y * nu);
    const int Y = offy + y, X = offx + x;
    dst[(long long)Y * nx + X] = src[stretch_src(Y, X, nx, rmap, cmap)];
  }
}

__global__ void k_stretch_full(const float* __restrict__ src, float* dst, const int* __restrict__ rmap,
                               const int* __restrict__ cmap, int nx, int ny) {
  const long long total = (long long)nx * ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int Y = (int)(t / nx), X = (int)(t - (long long)Y * nx);
    dst[t] = src[stretch_src(Y, X, nx, rmap, cmap)];
  }
}

int grid_for(long long items) { return (int)std::min<long long>((items + 255) / 256, 148LL * 8); }

}  // namespace

cudaError_t launch_stretch_crop(const void* const* slot, long long offset, const void* frame, int wl, void* dst,
                                const int* rmap, const int* cmap, int nx, int offx, int offy, int nu,
                                cudaStream_t st) {
  const int g = grid_for((long long)nu * nu);
  switch (wl) {
    case 1:
      k_stretch_crop<uint8_t><<<g, 256, 0, st>>>(slot, offset, frame, (uint8_t*)dst, rmap, cmap, nx, offx, offy, nu);
      break;
    case 2:
      k_stretch_crop<uint16_t><<<g, 256, 0, st>>>(slot, offset, frame, (uint16_t*)dst, rmap, cmap, nx, offx, offy,
                                                  nu);
      break;
    case 4:
      k_stretch_crop<uint32_t><<<g, 256, 0, st>>>(slot, offset, frame, (uint32_t*)dst, rmap, cmap, nx, offx, offy,
                                                  nu);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_stretch_full(const float* src, float* dst, const int* rmap, const int* cmap, int nx, int ny,
                                cudaStream_t st) {
  k_stretch_full<<<grid_for((long long)nx * ny), 256, 0, st>>>(src, dst, rmap, cmap, nx, ny);
  return cudaGetLastError();
}

}  // namespace mc
