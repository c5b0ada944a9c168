// Terrain preparation on the device: slope and aspect from a DEM.
//
// The reference takes slope and aspect from its terrain loader; this pass
// derives them from elevation so that a caller with only a DEM keeps its
// rasters on the GPU.  Gradients are central differences inside the grid and
// one-sided differences on its edges, in double precision from the float
// DEM; dx and dy are the signed cell sizes of the geo transform (dy < 0 for
// a north-up grid), so the row gradient is always the northward one.
//   slope  = |grad z| (rise over run)
//   aspect = compass azimuth of -grad z in [0, 2 pi), 0 where the ground is flat
#include <cuda_runtime.h>

#include <cstdint>

namespace propag {

__global__ void __launch_bounds__(256) slope_aspect_kernel(int W, int H, double dx, double dy,
                                                           const float *__restrict__ dem,
                                                           float *__restrict__ slope,
                                                           float *__restrict__ aspect) {
  const int64_t n = (int64_t)W * H;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % W), y = (int)(i / W);
    double gx = 0.0, gy = 0.0;
    if (W > 1) {
      if (x == 0) gx = ((double)__ldg(dem + i + 1) - (double)__ldg(dem + i)) / dx;
      else if (x == W - 1) gx = ((double)__ldg(dem + i) - (double)__ldg(dem + i - 1)) / dx;
      else gx = ((double)__ldg(dem + i + 1) - (double)__ldg(dem + i - 1)) / (2.0 * dx);
    }
    if (H > 1) {
      if (y == 0) gy = ((double)__ldg(dem + i + W) - (double)__ldg(dem + i)) / dy;
      else if (y == H - 1) gy = ((double)__ldg(dem + i) - (double)__ldg(dem + i - W)) / dy;
      else gy = ((double)__ldg(dem + i + W) - (double)__ldg(dem + i - W)) / (2.0 * dy);
    }
    const double s = hypot(gx, gy);
    double a = atan2(-gx, -gy);
    if (a < 0.0) a += 2.0 * 3.14159265358979323846;
    if (s == 0.0) a = 0.0;
    slope[i] = (float)s;
    aspect[i] = (float)a;
  }
}

cudaError_t launch_slope_aspect(int W, int H, double dx, double dy, const float *dem, float *slope,
                                float *aspect, int sm_count, cudaStream_t stream) {
  const uint64_t n = (uint64_t)W * H;
  uint64_t blocks = (n + 255) / 256;
  const uint64_t cap = (uint64_t)sm_count * 8;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  slope_aspect_kernel<<<(unsigned)blocks, 256, 0, stream>>>(W, H, dx, dy, dem, slope, aspect);
  return cudaGetLastError();
}

}  // namespace propag
