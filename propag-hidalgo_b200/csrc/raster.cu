// Input preparation on the device: rasterisation of ignition and fuel
// geometries, and the ignition list of a time raster.
//
// The reference burns its TimeFeatures and FuelFeatures into a raster with
// GDALRasterizeGeometries on the host (crates/propag/src/propag.rs:837-890,
// 929-982), features in order, later ones over earlier ones.  Here the host
// only parses the WKB and turns it into a pixel-space plan (raster.hpp); the
// work that grows with the grid runs on the device in three passes:
//   1. every cell of a winner raster (int32) is set to -1;
//   2. segment samples (one thread each) and polygon rows (one CTA each: the
//      row's edge crossings toggle bits of a shared-memory row mask, a prefix
//      XOR over the mask gives the even-odd inside test) raise the cells they
//      burn to their feature's index with atomicMax -- the largest index is
//      the last feature in burn order, whatever order the threads run in;
//   3. each cell takes its winner's value (a time, or a fuel code) or nodata.
// The same per-sample and per-edge functions as the host rasteriser give
// bit-identical rasters.  This file is compiled with -fmad=false.
#include <cuda_runtime.h>

#include <cstdint>

#include "raster_kernels.cuh"

namespace propag {
using namespace raster_dev;
namespace {

unsigned grid_for(uint64_t items, int sm_count, int per_sm) {
  uint64_t b = items;
  const uint64_t cap = (uint64_t)(sm_count > 0 ? sm_count : 1) * per_sm;
  if (b > cap) b = cap;
  return b == 0 ? 1u : (unsigned)b;
}

}  // namespace

cudaError_t launch_rasterize_winner(const RasterPlanDev &p, int64_t W, int64_t H, int32_t *win,
                                    int sm_count, cudaStream_t stream) {
  if (W < 1 || H < 1 || W > 32 * (int64_t)kRowWords) return cudaErrorInvalidValue;
  const int64_t n = W * H;
  fill_winner_kernel<<<grid_for(((uint64_t)n + kRasterThreads - 1) / kRasterThreads, sm_count, 8),
                       kRasterThreads, 0, stream>>>(win, n);
  if (p.samples)
    segment_kernel<<<grid_for((p.samples + kRasterThreads - 1) / kRasterThreads, sm_count, 8),
                     kRasterThreads, 0, stream>>>(p.segs, p.nseg, p.samples, W, H, win);
  if (p.rows)
    polygon_kernel<<<grid_for(p.rows, sm_count, 4), kRasterThreads, 0, stream>>>(
        p.polys, p.npoly, p.rows, p.edges, W, win);
  return cudaGetLastError();
}

cudaError_t launch_finish_times(float *times, const float *value, int64_t n, int sm_count,
                                cudaStream_t stream) {
  finish_times_kernel<<<grid_for(((uint64_t)n + kRasterThreads - 1) / kRasterThreads, sm_count, 8),
                        kRasterThreads, 0, stream>>>(times, value, n);
  return cudaGetLastError();
}

cudaError_t launch_finish_codes(const int32_t *win, const uint8_t *value, uint8_t *out, int64_t n,
                                int sm_count, cudaStream_t stream) {
  finish_codes_kernel<<<grid_for(((uint64_t)n + kRasterThreads - 1) / kRasterThreads, sm_count, 8),
                        kRasterThreads, 0, stream>>>(win, value, out, n);
  return cudaGetLastError();
}

uint64_t burning_chunks(int64_t n) { return ((uint64_t)n + kChunk - 1) / kChunk; }

// counts: burning_chunks(n) words; offsets: burning_chunks(n) + 1 words.
cudaError_t launch_burning_list(const float *times, int64_t W, int64_t H, uint32_t *counts,
                                uint64_t *offsets, PropagIgnition *out, uint64_t max_out,
                                int sm_count, cudaStream_t stream) {
  const int64_t n = W * H;
  const uint64_t chunks = burning_chunks(n);
  count_burning_kernel<<<grid_for(chunks, sm_count, 8), kRasterThreads, 0, stream>>>(times, n,
                                                                                    chunks, counts);
  scan_counts_kernel<<<1, 1024, 0, stream>>>(counts, chunks, offsets);
  write_burning_kernel<<<grid_for(chunks, sm_count, 8), kRasterThreads, 0, stream>>>(
      times, n, W, chunks, offsets, out, max_out);
  return cudaGetLastError();
}

}  // namespace propag
