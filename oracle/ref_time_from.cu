// TEST INFRASTRUCTURE ONLY -- the reference's own time_from on the GPU.
//
// This file holds no reference code: it includes the reference's kernel
// source (crates/propag/src/propag.cu, with crates/propag/src/propag.h)
// where it lies in the reference checkout, as oracle/Makefile's `ref` target
// compiles it, and evaluates Propagator::time_from (propag.cu:269-294) for a
// list of cases.  The build follows the reference's own
// (crates/propag/build.rs:48-69: nvcc -arch compute_80 -std=c++17 -O3, PTX
// that the driver compiles for the GPU at load time), so the arithmetic --
// CUDA's atan2f, __cosf, __frcp_rd, __fsqrt_rz and whatever multiply-adds
// nvcc contracts -- is the reference kernel's.  NDEBUG turns the reference's
// ASSERTs (device assert) off; the cases are valid inputs (eccentricity in
// [0, 1), speed > 0).  Only the harness kernel below is ever launched.
//
// Propagator derives the cell it evaluates from its launch geometry
// (index_2d, propag.h:82-87): with 64 blocks of 256 threads, grid_x = 1 and
// grid_y = Y, thread g evaluates cell (16384 + g, Y).  A case gives the
// source cell as an offset from that cell.
#include <assert.h>
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

// time_from is a private member of the reference's Propagator
#define private public
#include "propag.cu"
#undef private

static constexpr int kThreads = 256, kBlocks = 64, kCasesPerLaunch = kThreads * kBlocks;
static constexpr int kToX0 = kCasesPerLaunch;  // the cell of thread g is (kToX0 + g, kToY)
static constexpr unsigned kToY = 16384;

__global__ void ref_time_from_kernel(const Settings settings, int64_t base, int64_t n,
                                     const int32_t *ddx, const int32_t *ddy, const float *ftime,
                                     const float *smax, const float *azmax, const float *ecc,
                                     float *out) {
  const int64_t g = threadIdx.x + (int64_t)blockIdx.x * blockDim.x;
  const int64_t i = base + g;
  if (i >= n) return;
  Propagator sim(settings, 1u, kToY, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  const int2 from = make_int2(kToX0 + (int)g + ddx[i], (int)kToY + ddy[i]);
  const PointRef ref(ftime[i], from);
  FireSimpleCuda fire;
  fire.speed_max = smax[i];
  fire.azimuth_max = azmax[i];
  fire.eccentricity = ecc[i];
  out[i] = sim.time_from(ref, fire);
}

// Evaluates n cases; case i goes from cell (to_x[i] + ddx[i], to_y[i] +
// ddy[i]) to cell (to_x[i], to_y[i]) (both written here), on a grid of pixel
// size (dx, dy), dy < 0 = north-up.  |ddx|, |ddy| <= 16383.  Returns 0 or the
// CUDA error code.
extern "C" int ref_time_from_batch(int64_t n, const int32_t *ddx, const int32_t *ddy,
                                   const float *ftime, const float *smax, const float *azmax,
                                   const float *ecc, float dx, float dy, float *out, int32_t *to_x,
                                   int32_t *to_y) {
  for (int64_t i = 0; i < n; ++i) {
    if (ddx[i] < -16383 || ddx[i] > 16383 || ddy[i] < -16383 || ddy[i] > 16383) return -1;
    to_x[i] = kToX0 + (int32_t)(i % kCasesPerLaunch);
    to_y[i] = (int32_t)kToY;
  }
  if (n == 0) return 0;
  Settings s;
  memset(&s, 0, sizeof(s));
  s.geo_ref.width = 65535;
  s.geo_ref.height = 65535;
  s.geo_ref.transform.gt.dx = dx;
  s.geo_ref.transform.gt.dy = dy;
  s.max_time = FLT_MAX;
  const size_t b = (size_t)n * 4;
  char *d = nullptr;
  cudaError_t e = cudaMalloc(&d, 7 * b);
  if (e != cudaSuccess) return (int)e;
  const void *src[6] = {ddx, ddy, ftime, smax, azmax, ecc};
  for (int k = 0; k < 6 && e == cudaSuccess; ++k)
    e = cudaMemcpy(d + k * b, src[k], b, cudaMemcpyHostToDevice);
  for (int64_t base = 0; base < n && e == cudaSuccess; base += kCasesPerLaunch) {
    ref_time_from_kernel<<<kBlocks, kThreads>>>(
        s, base, n, (const int32_t *)d, (const int32_t *)(d + b), (const float *)(d + 2 * b),
        (const float *)(d + 3 * b), (const float *)(d + 4 * b), (const float *)(d + 5 * b),
        (float *)(d + 6 * b));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + 6 * b, b, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}
