// The rasterisation kernels (see raster.cu for the passes and the host
// side).  Kept in a header of their own so that the CPU tests can compile
// the same source for the host, with the CUDA built-ins replaced by a
// thread-level emulation (tests/emul/).
#pragma once

#include <cfloat>
#include <cstdint>

#include "propag_b200.h"
#include "raster.hpp"

namespace propag {
namespace raster_dev {

constexpr int kRasterThreads = 256;  // every kernel below assumes 8 warps
constexpr int kRowWords = 2048;      // row mask words: 65536 columns

__global__ void __launch_bounds__(kRasterThreads) fill_winner_kernel(int32_t *win, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    win[i] = -1;
}

// The index of the last part whose `before` is <= i (`before` strictly
// increasing from 0).
template <typename T>
__device__ __forceinline__ uint64_t find_part(const T *parts, uint64_t n, uint64_t i) {
  uint64_t lo = 0, hi = n - 1;
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo + 1) / 2;
    if (parts[mid].before <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(kRasterThreads)
    segment_kernel(const RasterSeg *__restrict__ segs, uint64_t nseg, uint64_t samples, int64_t W,
                   int64_t H, int32_t *__restrict__ win) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < samples;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const RasterSeg &g = segs[find_part(segs, nseg, i)];
    const int64_t s = g.s0 + (int64_t)(i - g.before);
    int64_t c, r;
    if (seg_sample(g, s, W, H, c, r)) atomicMax(win + r * W + c, g.feature);
  }
}

// One polygon row per CTA iteration.  W <= 32 * kRowWords.
__global__ void __launch_bounds__(kRasterThreads)
    polygon_kernel(const RasterPoly *__restrict__ polys, uint64_t npoly, uint64_t rows,
                   const RasterEdge *__restrict__ edges, int64_t W, int32_t *__restrict__ win) {
  __shared__ uint32_t mask[kRowWords];
  __shared__ uint32_t warp_parity[kRasterThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nw = (int)((W + 31) / 32);
  const int per = (nw + kRasterThreads - 1) / kRasterThreads;  // words per thread
  const int w0 = min(nw, tid * per), w1 = min(nw, w0 + per);
  for (uint64_t item = blockIdx.x; item < rows; item += gridDim.x) {
    const RasterPoly p = polys[find_part(polys, npoly, item)];
    const int64_t r = (int64_t)p.row0 + (int64_t)(item - p.before);
    for (int w = tid; w < nw; w += kRasterThreads) mask[w] = 0u;
    __syncthreads();
    // a crossing toggles the first column whose centre is at or right of it
    const double yc = (double)r + 0.5;
    for (uint64_t k = tid; k < p.count; k += kRasterThreads) {
      double x;
      if (!edge_crossing(edges[p.first + k], yc, x)) continue;
      const int64_t c = crossing_cell(x, W);
      if (c < W) atomicXor(&mask[c >> 5], 1u << (c & 31));
    }
    __syncthreads();
    // inside = odd number of toggles at or left of the column: an inclusive
    // prefix XOR along the row (within a word by shifts, across words and
    // threads by the parity of everything ahead)
    uint32_t par = 0;
    for (int w = w0; w < w1; ++w) par ^= (uint32_t)__popc(mask[w]) & 1u;
    const uint32_t vote = __ballot_sync(0xFFFFFFFFu, par != 0u);
    uint32_t carry = (uint32_t)__popc(vote & ((1u << lane) - 1u)) & 1u;
    if (lane == 0) warp_parity[wid] = (uint32_t)__popc(vote) & 1u;
    __syncthreads();
    for (int k = 0; k < wid; ++k) carry ^= warp_parity[k];
    for (int w = w0; w < w1; ++w) {
      const uint32_t b = mask[w];
      uint32_t m = b;
      m ^= m << 1;
      m ^= m << 2;
      m ^= m << 4;
      m ^= m << 8;
      m ^= m << 16;
      mask[w] = carry ? ~m : m;
      carry ^= (uint32_t)__popc(b) & 1u;
    }
    __syncthreads();
    int32_t *row = win + r * W;
    for (int64_t c = tid; c < W; c += kRasterThreads)
      if ((mask[c >> 5] >> (c & 31)) & 1u) atomicMax(row + c, p.feature);
    __syncthreads();  // the mask is reused by the next row
  }
}

// In place: the winner raster (int32 in the float buffer) becomes times.
__global__ void __launch_bounds__(kRasterThreads)
    finish_times_kernel(float *times, const float *__restrict__ value, int64_t n) {
  int32_t *win = reinterpret_cast<int32_t *>(times);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t w = win[i];
    times[i] = w >= 0 ? value[w] : FLT_MAX;
  }
}

__global__ void __launch_bounds__(kRasterThreads)
    finish_codes_kernel(const int32_t *__restrict__ win, const uint8_t *__restrict__ value,
                        uint8_t *__restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t w = win[i];
    out[i] = w >= 0 ? value[w] : (uint8_t)255;
  }
}

// ---- ignition list of a time raster ------------------------------------------
constexpr int kChunk = 4096;  // cells per CTA iteration of the count and write passes

__global__ void __launch_bounds__(kRasterThreads)
    count_burning_kernel(const float *__restrict__ t, int64_t n, uint64_t chunks,
                         uint32_t *__restrict__ counts) {
  __shared__ uint32_t part[kRasterThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint64_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
    const int64_t base = (int64_t)ch * kChunk;
    uint32_t k = 0;
    for (int j = threadIdx.x; j < kChunk; j += kRasterThreads) {
      const int64_t i = base + j;
      if (i < n && t[i] != FLT_MAX) ++k;
    }
    for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xFFFFFFFFu, k, o);
    if (lane == 0) part[wid] = k;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t s = 0;
      for (int w = 0; w < kRasterThreads / 32; ++w) s += part[w];
      counts[ch] = s;
    }
    __syncthreads();
  }
}

// One CTA: offsets[k] = sum of counts[0 .. k), offsets[chunks] = the total.
__global__ void __launch_bounds__(1024)
    scan_counts_kernel(const uint32_t *__restrict__ counts, uint64_t chunks,
                       uint64_t *__restrict__ offsets) {
  __shared__ uint64_t part[1024];
  const uint64_t per = (chunks + blockDim.x - 1) / blockDim.x;
  const uint64_t a = min(chunks, (uint64_t)threadIdx.x * per), b = min(chunks, a + per);
  uint64_t s = 0;
  for (uint64_t k = a; k < b; ++k) s += counts[k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (unsigned d = 1; d < blockDim.x; d <<= 1) {
    const uint64_t v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint64_t run = part[threadIdx.x] - s;
  for (uint64_t k = a; k < b; ++k) {
    offsets[k] = run;
    run += counts[k];
  }
  if (threadIdx.x == blockDim.x - 1) offsets[chunks] = part[threadIdx.x];
}

// Burning cells (time != FLT_MAX, NaN included) in row-major order.
__global__ void __launch_bounds__(kRasterThreads)
    write_burning_kernel(const float *__restrict__ t, int64_t n, int64_t W, uint64_t chunks,
                         const uint64_t *__restrict__ offsets, PropagIgnition *__restrict__ out,
                         uint64_t max_out) {
  __shared__ uint32_t warp_count[kRasterThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint64_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
    uint64_t at = offsets[ch];
    const int64_t base = (int64_t)ch * kChunk;
    for (int j0 = 0; j0 < kChunk; j0 += kRasterThreads) {
      const int64_t i = base + j0 + threadIdx.x;
      const float v = i < n ? t[i] : FLT_MAX;
      const bool hit = v != FLT_MAX;
      const uint32_t vote = __ballot_sync(0xFFFFFFFFu, hit);
      if (lane == 0) warp_count[wid] = (uint32_t)__popc(vote);
      __syncthreads();
      uint32_t ahead = (uint32_t)__popc(vote & ((1u << lane) - 1u)), total = 0;
      for (int w = 0; w < kRasterThreads / 32; ++w) {
        if (w < wid) ahead += warp_count[w];
        total += warp_count[w];
      }
      if (hit && at + ahead < max_out) {
        PropagIgnition g;
        g.x = (uint32_t)(i % W);
        g.y = (uint32_t)(i / W);
        g.time = v;
        out[at + ahead] = g;
      }
      at += total;
      __syncthreads();  // warp_count is rewritten by the next step
    }
  }
}

}  // namespace raster_dev
}  // namespace propag
