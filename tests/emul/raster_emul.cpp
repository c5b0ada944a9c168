// Test infrastructure: the rasterisation kernels (raster_kernels.cuh, the
// same source the device build compiles) run on the host by
// cuda_host_emul.hpp, behind the same passes as the launchers in raster.cu.
// Built by tests/test_raster_kernels_emulated.py with g++ -std=c++20.
#include "cuda_host_emul.hpp"
#include "raster_kernels.cuh"
#include "io.hpp"

using namespace propag;
using namespace propag::raster_dev;

namespace {

template <typename GetWkb>
RasterPlan plan_of(const GeoReference &g, uint64_t n, GetWkb &&wkb) {
  RasterPlan plan;
  for (uint64_t i = 0; i < n; ++i) {
    const uint8_t *d = nullptr;
    uintptr_t l = 0;
    wkb(i, d, l);
    if (!d || l == 0) continue;
    Geometry geom;
    if (!parse_wkb(d, l, geom)) continue;
    plan_geometry(g, geom, (int32_t)i, plan);
  }
  return plan;
}

void winner(const RasterPlan &plan, int64_t W, int64_t H, int32_t *win, unsigned grid) {
  emul::launch(grid, kRasterThreads, fill_winner_kernel, win, W * H);
  if (plan.samples)
    emul::launch(grid, kRasterThreads, segment_kernel, (const RasterSeg *)plan.segs.data(),
                 (uint64_t)plan.segs.size(), plan.samples, W, H, win);
  if (plan.rows)
    emul::launch(grid, kRasterThreads, polygon_kernel, (const RasterPoly *)plan.polys.data(),
                 (uint64_t)plan.polys.size(), plan.rows, (const RasterEdge *)plan.edges.data(), W, win);
}

}  // namespace

extern "C" int emul_rasterize_times(const GeoReference *g, const FFITimeFeature *f, uint64_t n,
                                    float *times, unsigned grid) {
  const RasterPlan plan = plan_of(*g, n, [&](uint64_t i, const uint8_t *&d, uintptr_t &l) {
    d = f[i].geom_wkb;
    l = f[i].geom_wkb_len;
  });
  std::vector<float> value(n);
  for (uint64_t i = 0; i < n; ++i) value[i] = f[i].time;
  const int64_t W = g->width, H = g->height;
  winner(plan, W, H, reinterpret_cast<int32_t *>(times), grid);
  emul::launch(grid, kRasterThreads, finish_times_kernel, times, (const float *)value.data(), W * H);
  return 0;
}

extern "C" int emul_rasterize_fuels(const FFIFuelFeature *f, uint64_t n, const GeoReference *g,
                                    uint8_t *out, unsigned grid) {
  const RasterPlan plan = plan_of(*g, n, [&](uint64_t i, const uint8_t *&d, uintptr_t &l) {
    d = f[i].geom_wkb;
    l = f[i].geom_wkb_len;
  });
  std::vector<uint8_t> value(n);
  for (uint64_t i = 0; i < n; ++i) value[i] = f[i].code;
  const int64_t W = g->width, H = g->height;
  std::vector<int32_t> win((size_t)(W * H));
  winner(plan, W, H, win.data(), grid);
  emul::launch(grid, kRasterThreads, finish_codes_kernel, (const int32_t *)win.data(),
               (const uint8_t *)value.data(), out, W * H);
  return 0;
}

extern "C" int64_t emul_ignitions_from_times(const float *t, uint32_t W, uint32_t H,
                                             PropagIgnition *out, uint64_t max_out, unsigned grid) {
  const int64_t n = (int64_t)W * H;
  const uint64_t chunks = ((uint64_t)n + kChunk - 1) / kChunk;
  std::vector<uint32_t> counts(chunks);
  std::vector<uint64_t> offsets(chunks + 1);
  emul::launch(grid, kRasterThreads, count_burning_kernel, t, n, chunks, counts.data());
  emul::launch(1, 1024, scan_counts_kernel, (const uint32_t *)counts.data(), chunks, offsets.data());
  emul::launch(grid, kRasterThreads, write_burning_kernel, t, n, (int64_t)W, chunks,
               (const uint64_t *)offsets.data(), out, max_out);
  return (int64_t)offsets[chunks];
}
